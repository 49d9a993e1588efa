"""Learned preconditioner: set-up on a matrix, training data from the plain solver, training on
the GPU, and the packaged weights.

The network (cstfem_b200.h, "learned preconditioner") maps a residual r to
z = D^-1 (r + s Y(r / s)); with the output layer at zero it is exactly the Jacobi step, which
is where training starts. Training pairs (r_k, e_k) come from plain FP64 Jacobi-PCG runs on
seeded random plates (the uneven batch distribution): r_k = b - A x_k and e_k = x* - x_k for
iterates x_k sampled along the run and x* the converged solution. The loss of a pair is the
squared sine of the energy-norm angle between z = M(r_k) and e_k (0 when z points along the
error). Forward, loss and backward run in the library's kernels; Adam runs on the GPU.

The same network also serves as the finest-level post-smoother of the multigrid cycle
(preconditioner "learned_mg"): the cycle's Chebyshev pre-smoothing and coarse correction give it
global reach, and the network maps the remaining residual r2 to omega D^-1 (r2 + s Y(r2 / s)),
omega = 4 / (3 lambda_max(D^-1 A)); with the output layer at zero it is one damped-Jacobi
post-smoothing step. It is trained on the same pairs with the loss of the whole cycle's output
(`--mode cycle`); its weights ship separately.

Command line (writes the packaged weights):
    python -m mpi-cst-fem-solver_b200.learned train --mode local|cycle --out weights.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import os
import time

import numpy as np

from . import native
from .native import CstgError
from .plate import PlateSpec, quarter_plate, random_batch, symmetry_dirichlet
from .solver import (CgJacobiSolver, Context, GpuCsrMatrix, PlaneCondition, SolverOptions, _f64, _ptr,
                     add_traction, apply_dirichlet, assemble_stiffness, build_stiffness_pattern,
                     constitutive_matrix)

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "mpnn_plates.npz")
WEIGHTS_CYCLE = os.path.join(HERE, "weights", "mpnn_cycle_smoother.npz")
N_PARAMS = 25474
F, N_IN, N_LAYERS = 64, 8, 3


def param_count() -> int:
    return int(native.load().cstg_mpnn_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal hidden weights, zero biases and a zero output layer (the network starts as
    the Jacobi step)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    o = 0
    p[o:o + F * N_IN] = rng.standard_normal(F * N_IN) * np.sqrt(2.0 / N_IN)
    o += F * N_IN + F
    for _ in range(N_LAYERS):
        # small residual branches: the hidden state grows slowly through the layers
        p[o:o + F * 2 * F] = rng.standard_normal(F * 2 * F) * np.sqrt(2.0 / (2 * F)) * 0.5
        o += F * 2 * F + F
    assert o + 2 * F + 2 == N_PARAMS
    return p


def node_material(D, n_nodes: int) -> np.ndarray:
    """The two material inputs per node: log(D00) and D01 / D00 of the constitutive matrix."""
    D = np.asarray(D, dtype=np.float64).reshape(-1, 9)
    if D.shape[0] == 1:
        D = np.repeat(D, n_nodes, axis=0)
    return np.ascontiguousarray(np.stack([np.log(D[:, 0]), D[:, 1] / D[:, 0]], axis=1).reshape(-1),
                                dtype=np.float32)


def load_weights(path: str | None = None, mode: str = "local") -> np.ndarray:
    """The packaged weights of the network alone (mode "local") or of the cycle's post-smoother
    ("cycle")."""
    path = path or (WEIGHTS if mode == "local" else WEIGHTS_CYCLE)
    if not os.path.exists(path):
        raise CstgError(native.ERR_STATE, f"learned preconditioner weights not found: {path}")
    p = np.load(path)["params"].astype(np.float32)
    if p.size != N_PARAMS:
        raise CstgError(native.ERR_INVALID_ARGUMENT, f"weights have {p.size} values, expected {N_PARAMS}")
    return p


def setup(K: GpuCsrMatrix, params: np.ndarray, material: np.ndarray) -> None:
    """cstg_learned_setup on K's context (after the Jacobi set-up of K)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    m = np.ascontiguousarray(material, dtype=np.float32)
    K.ctx.check(K.ctx.L.cstg_learned_setup(K.ctx.h, _ptr(p), _ptr(m)))


def apply(K: GpuCsrMatrix, r, z=None):
    """z = M(r) on CUDA float64 tensors."""
    import torch
    z = torch.empty_like(r) if z is None else z
    with K.ctx.ordered(r.device):
        K.ctx.check(K.ctx.L.cstg_learned_apply_device(K.ctx.h, _ptr(r), _ptr(z)))
    return z


def time_stages(K: GpuCsrMatrix, reps: int = 20) -> dict:
    """Seconds per launch of the encoder and of each message-passing layer (cstg_learned_time)."""
    out = (C.c_double * 4)()
    K.ctx.check(K.ctx.L.cstg_learned_time(K.ctx.h, int(reps), out))
    return {"encoder_s": out[0], "layer_s": [out[1], out[2], out[3]]}


def cycle_parts(K: GpuCsrMatrix, r) -> dict:
    """The learned cycle's parts for the CUDA float64 residual r: x_fix (pre-smoothing + coarse
    correction), r2 = r - A x_fix, winvd = omega D^-1 and the cycle's output z."""
    import torch
    out = {k: torch.empty_like(r) for k in ("xfix", "r2", "winvd", "z")}
    with K.ctx.ordered(r.device):
        K.ctx.check(K.ctx.L.cstg_learned_cycle_parts_device(K.ctx.h, _ptr(r), _ptr(out["xfix"]), _ptr(out["r2"]),
                                                            _ptr(out["winvd"]), _ptr(out["z"])))
    return out


class Trainer:
    """The GPU trainer (cstg_trainer): FP32 master weights + Adam state on the device."""

    def __init__(self, params: np.ndarray, device: int = 0):
        self.L = native.load()
        st = C.c_int(0)
        p = np.ascontiguousarray(params, dtype=np.float32)
        self.h = self.L.cstg_trainer_create(device, _ptr(p), C.byref(st))
        if not self.h:
            raise CstgError(st.value, f"cstg_trainer_create failed (status {st.value})")

    def _check(self, rc):
        if rc:
            raise CstgError(rc, self.L.cstg_trainer_last_error(self.h).decode())

    def accumulate(self, K: GpuCsrMatrix, R, E) -> np.ndarray:
        """Adds the gradients of the samples (rows of the CUDA float64 tensors R, E)."""
        ns = int(R.shape[0])
        losses = np.zeros(ns)
        R, E = R.contiguous(), E.contiguous()
        with K.ctx.ordered(R.device):  # (the trainer starts by waiting for the context's stream)
            self._check(self.L.cstg_trainer_accumulate(self.h, K.ctx.h, ns, _ptr(R), _ptr(E), _ptr(losses)))
        return losses

    def accumulate_cycle(self, K: GpuCsrMatrix, R, E) -> np.ndarray:
        """As accumulate, with the network as the multigrid cycle's post-smoother and the loss of
        the whole cycle's output."""
        ns = int(R.shape[0])
        losses = np.zeros(ns)
        R, E = R.contiguous(), E.contiguous()
        with K.ctx.ordered(R.device):
            self._check(self.L.cstg_trainer_accumulate_cycle(self.h, K.ctx.h, ns, _ptr(R), _ptr(E), _ptr(losses)))
        return losses

    def step(self, lr: float, grad_scale: float) -> None:
        self._check(self.L.cstg_trainer_step(self.h, float(lr), float(grad_scale)))

    def params(self, grads: bool = False):
        p = np.zeros(N_PARAMS, dtype=np.float32)
        g = np.zeros(N_PARAMS, dtype=np.float32) if grads else None
        self._check(self.L.cstg_trainer_params(self.h, _ptr(p), _ptr(g)))
        return (p, g) if grads else p

    def zero_grad(self) -> None:
        self._check(self.L.cstg_trainer_zero_grad(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.cstg_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class PlateProblem:
    """One training plate on the GPU: its matrix (learned set-up done) and sample pairs."""
    spec: PlateSpec
    K: GpuCsrMatrix
    R: object  # CUDA float64 [samples, n]
    E: object


def plate_system(spec: PlateSpec, ctx: Context | None = None, load=("right", 1.0, 0.0)):
    """Assembled, eliminated plate and its right-hand side (host b)."""
    m = quarter_plate(spec.n_r, spec.n_theta, a=spec.a)
    D = constitutive_matrix(spec.E, spec.nu, PlaneCondition.Strain if spec.plane_strain else PlaneCondition.Stress)
    K = build_stiffness_pattern(m, ctx=ctx)
    assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    add_traction(K, m.boundary_edges[load[0]], 1.0, load[1], load[2], b)
    apply_dirichlet(symmetry_dirichlet(m), K, b)
    return m, D, K, b


def harvest(spec: PlateSpec, samples: int, params: np.ndarray, seed: int = 0, device: int = 0) -> PlateProblem:
    """Training pairs from plain FP64 Jacobi-PCG on one plate (a random load case mix)."""
    import torch
    rng = np.random.default_rng(seed)
    ctx = Context(device)
    loads = [("right", 1.0, 0.0), ("top", 0.0, 1.0), ("right", 0.0, 1.0), ("top", 1.0, 0.0)]
    m, D, K, b = plate_system(spec, ctx, loads[int(rng.integers(0, 4))])
    s = CgJacobiSolver(SolverOptions(rtol=1e-12, max_iter=200000))
    s.setup(K)
    d_b = torch.from_numpy(b).to(device)
    x_star = torch.zeros_like(d_b)
    st = s.solve(d_b, x_star)
    if not st.converged:
        raise CstgError(native.ERR_STATE, f"harvest: reference solve failed: {st.message}")
    iters = max(st.iterations, samples)
    every = max(1, iters // (samples + 1))
    X = torch.zeros((samples, m.num_dofs), dtype=torch.float64, device=device)
    o = SolverOptions(rtol=1e-12, max_iter=200000).native()
    got = C.c_int(0)
    stats = native.Stats()
    with ctx.ordered(d_b.device):
        ctx.check(ctx.L.cstg_pcg_iterates_device(ctx.h, _ptr(d_b), every, samples, _ptr(X), C.byref(got),
                                                 C.byref(o), C.byref(stats)))
    X = X[:got.value]
    E = (x_star[None, :] - X).contiguous()
    R = torch.empty_like(E)
    for i in range(E.shape[0]):
        R[i] = d_b - K.multiply(X[i].contiguous())
    keep = torch.linalg.vector_norm(R, dim=1) > 1e-9 * torch.linalg.vector_norm(d_b)
    R, E = R[keep].contiguous(), E[keep].contiguous()
    setup(K, params, node_material(D, m.num_nodes))
    return PlateProblem(spec=spec, K=K, R=R, E=E)


def train(n_plates: int = 100, samples_per_plate: int = 100, epochs: int = 3, batch: int = 8, lr: float = 1e-3,
          seed: int = 2026, n_r_range=(20, 200), device: int = 0, log=print, mode: str = "local"):
    """Harvests n_plates x samples_per_plate pairs from the uneven plate distribution and trains
    the network (mode "local": the network alone; "cycle": as the multigrid cycle's
    post-smoother); returns (params, history of mean epoch losses, number of pairs)."""
    if mode not in ("local", "cycle"):
        raise ValueError(f"train: unknown mode {mode!r}")
    import torch
    params0 = init_params(seed)
    specs = random_batch(count=n_plates, seed=seed + 1, n_r_range=n_r_range)
    t0 = time.perf_counter()
    probs = [harvest(sp, samples_per_plate, params0, seed=seed + 7 * i, device=device) for i, sp in enumerate(specs)]
    n_pairs = sum(int(p.R.shape[0]) for p in probs)
    log(f"harvested {n_pairs} pairs from {n_plates} plates in {time.perf_counter() - t0:.1f} s")
    tr = Trainer(params0, device)
    rng = np.random.default_rng(seed + 3)
    hist = []
    start = None
    for ep in range(epochs):
        order = [(i, j) for i, p in enumerate(probs) for j in range(0, int(p.R.shape[0]), batch)]
        rng.shuffle(order)
        tot, cnt = 0.0, 0
        t1 = time.perf_counter()
        for i, j in order:
            p = probs[i]
            Rb, Eb = p.R[j:j + batch], p.E[j:j + batch]
            losses = tr.accumulate(p.K, Rb, Eb) if mode == "local" else tr.accumulate_cycle(p.K, Rb, Eb)
            if not np.all(np.isfinite(losses)):
                tr.zero_grad()
                continue
            tr.step(lr, 1.0 / len(losses))
            tot += float(losses.sum())
            cnt += len(losses)
        mean = tot / max(cnt, 1)
        if start is None:
            start = mean
        hist.append(mean)
        log(f"epoch {ep}: mean loss {mean:.5f} ({time.perf_counter() - t1:.1f} s)")
    params = tr.params()
    tr.close()
    for p in probs:
        p.K.ctx.close()
    return params, hist, n_pairs


def scale_output(params: np.ndarray, gain: float) -> np.ndarray:
    """The network with its output layer (W_out, b_out) multiplied by `gain`."""
    p = np.array(params, dtype=np.float32, copy=True)
    p[-(2 * F + 2):] *= np.float32(gain)
    return p


def select_gain(params: np.ndarray, n_plates: int = 8, seed: int = 5151, gains=(0.25, 0.5, 0.75, 1.0),
                n_r_range=(60, 160), device: int = 0, log=print):
    """Chooses the output gain of the cycle's post-smoother on validation plates (seeded draws
    from the training distribution, not the training batch). The network's output varies
    nonlinearly with r: a full-strength correction lowers the per-step loss most but can cost
    Krylov iterations, so the gain is chosen on the solve itself, against the same cycle with the
    network at zero (gain 0): the gain whose worst plate (iterations / iterations at gain 0) is
    lowest, ties broken by the total. Returns (gain, {gain: [iterations per plate]})."""
    from .solver import CgJacobiSolver, SolverOptions
    specs = random_batch(count=n_plates, seed=seed, n_r_range=n_r_range)
    systems = [plate_system(spec, Context(device)) for spec in specs]
    its = {}
    for g in (0.0,) + tuple(gains):
        p = scale_output(params, g)
        row = []
        for m, D, K, b in systems:
            s = CgJacobiSolver(SolverOptions(rtol=1e-10, max_iter=5000, precision="mixed",
                                             preconditioner="learned_mg", true_residual_stop=True))
            s.setup(K)
            setup(K, p, node_material(D, m.num_nodes))
            st = s.solve(b, np.zeros(m.num_dofs))
            row.append(st.iterations if st.converged else 10 ** 6)
        its[float(g)] = row
        log(f"gain {g}: iterations {row} (total {sum(row)})")
    for m, D, K, b in systems:
        K.ctx.close()
    base = np.array(its[0.0], dtype=float)

    def score(g):
        r = np.array(its[g], dtype=float) / base
        return (float(r.max()), sum(its[g]))
    best = min((g for g in its if g > 0.0), key=score)
    return best, its


def gain_record(raw: np.ndarray) -> dict:
    """select_gain on the raw (unscaled) parameters, as fields of the weights file."""
    gain, its = select_gain(raw)
    print(f"output gain {gain} (validation iterations {its})")
    return dict(output_gain=gain, params_raw=raw,
                gain_iterations=np.array([[g] + list(v) for g, v in sorted(its.items())], dtype=np.float64))


def main():
    ap = argparse.ArgumentParser(description="train the learned preconditioner on the GPU")
    ap.add_argument("cmd", choices=["train", "select-gain"])
    ap.add_argument("--mode", choices=["local", "cycle"], default="local")
    ap.add_argument("--out", default=None)
    ap.add_argument("--plates", type=int, default=100)
    ap.add_argument("--samples", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--n-r-max", type=int, default=200)
    a = ap.parse_args()
    out = a.out or (WEIGHTS if a.mode == "local" else WEIGHTS_CYCLE)
    if a.cmd == "select-gain":  # re-select the cycle smoother's output gain of a weights file
        d = dict(np.load(WEIGHTS_CYCLE))
        raw = d["params_raw"] if "params_raw" in d else scale_output(d["params"], 1.0 / float(d["output_gain"]))
        d.update(gain_record(raw.astype(np.float32)))
        d["params"] = scale_output(raw, float(d["output_gain"]))
        np.savez(out, **d)
        print(f"wrote {out}")
        return
    t0 = time.perf_counter()
    params, hist, n_pairs = train(a.plates, a.samples, a.epochs, a.batch, a.lr, a.seed, (20, a.n_r_max),
                                  mode=a.mode)
    extra = {}
    if a.mode == "cycle":
        extra = gain_record(params)
        params = scale_output(params, float(extra["output_gain"]))
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.savez(out, params=params, loss_history=np.array(hist), pairs=n_pairs, plates=a.plates,
             samples=a.samples, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, mode=a.mode,
             seconds=time.perf_counter() - t0, **extra)
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
