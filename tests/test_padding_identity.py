"""The network layers sum each node's neighbour rows in FP32 over a fixed number of slots, padding
the slots past the node's degree with rows of BF16 -0.0 (csrc/mpnn.cu, k_mp_layer_ws and
k_mp_layer_tc): the sum keeps the bits of the sum over the real neighbours only because
x + (-0) = x exactly in IEEE round-to-nearest for every x, both zeros included. The mean's
1/deg comes from a table of the IEEE quotients 1.f / d (constants folded by the compiler). This
checks both facts on the CPU in numpy FP32, over values spanning the exponent range, signed zeros,
subnormals and infinities."""
import numpy as np


def _bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def test_negative_zero_is_an_exact_additive_identity():
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(200000) * np.exp2(rng.integers(-140, 120, 200000))).astype(np.float32)
    x = np.concatenate([x, np.float32([0.0, -0.0, 1e-45, -1e-45, 1.17e-38, np.inf, -np.inf, 3.4e38])])
    nz = np.float32(-0.0)
    assert np.array_equal(_bits(x + nz), _bits(x))
    # a padded chain of adds equals the unpadded chain bit for bit, wherever the padding falls
    terms = (rng.standard_normal((1000, 6)) * 10.0).astype(np.float32)
    for k in range(7):
        acc, acc_pad = np.zeros(1000, np.float32), np.zeros(1000, np.float32)
        for j in range(6):
            acc = acc + terms[:, j]
        for j in range(7):
            acc_pad = acc_pad + (nz if j == k else terms[:, j - (j > k)])
        assert np.array_equal(_bits(acc), _bits(acc_pad)), k
    # (+0 would not do: -0 + +0 = +0 changes the sign of a sum that is -0)
    assert _bits(np.float32(-0.0) + np.float32(0.0)) != _bits(np.float32(-0.0))


def test_inverse_degree_table_is_the_ieee_quotient():
    for d in range(1, 8):
        q = np.float32(1.0) / np.float32(d)  # IEEE round-to-nearest quotient
        exact = 1.0 / d
        # the correctly rounded value: no other FP32 is nearer to 1/d
        nxt = np.nextafter(q, np.float32(1.0), dtype=np.float32)
        prv = np.nextafter(q, np.float32(0.0), dtype=np.float32)
        assert abs(float(q) - exact) <= min(abs(float(nxt) - exact), abs(float(prv) - exact))
