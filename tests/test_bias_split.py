"""The network kernels add each FP32 bias inside the tensor-core product: the bias b enters as
three BF16 parts against constant ones in the A operand, b_hi = bf16(b), b_mid = bf16(b - b_hi),
b_lo = bf16(b - b_hi - b_mid) (csrc/mpnn.cu, k_mp_encode and k_mp_layer_tc). This checks on the
CPU, with BF16 round-to-nearest-even emulated in numpy, that both differences are exact in FP32
and that the three parts sum to b exactly, over FP32 values spanning 26 decades."""
import numpy as np


def _bf16(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def test_three_part_bf16_split_is_exact():
    rng = np.random.default_rng(7)
    n = 200_000
    b = (rng.standard_normal(n) * np.exp(rng.uniform(-30.0, 30.0, n))).astype(np.float32)
    b = np.concatenate([b, np.float32([0.0, 1.0, -1.0, 3.1415927, 1e-20, -7.5e12])])
    hi = _bf16(b)
    r1 = (b - hi).astype(np.float32)
    mid = _bf16(r1)
    r2 = (r1 - mid).astype(np.float32)
    lo = _bf16(r2)
    f64 = np.float64
    assert np.array_equal(b.astype(f64) - hi.astype(f64), r1.astype(f64))
    assert np.array_equal(r1.astype(f64) - mid.astype(f64), r2.astype(f64))
    assert np.array_equal(hi.astype(f64) + mid.astype(f64) + lo.astype(f64), b.astype(f64))
