"""Golden fixtures at the benchmark sizes, computed by the reference's own serial core.

The reference's path (build_stiffness_pattern -> assemble_stiffness -> add_traction ->
apply_dirichlet -> CgJacobiSolver at rtol 1e-10, src/assembly.cpp, src/bc.cpp,
src/solver.cpp) is run to convergence on two O-grid quarter plates:

* 400 x 1250 (1,003,302 DOFs: the literal refined plate of the benchmark family);
* 565 x 1766 (2,000,244 DOFs: the size-corrected 2M-DOF plate the benchmark times).

Per plate it writes `plate_<n_r>x<n_theta>.json` with SHA-256 digests of the mesh, the CSR
pattern, K, K after the Dirichlet elimination, the load vector before and after it, the
solver's outcome (iterations, recursive and true relative residual), the stress concentration
factor at the hole, and the wall-clock time of every phase on this host (the measured CPU
baseline: one core, the reference is single-threaded). The `.npz` beside it holds the
displacements: all of them for the 1M-DOF plate, every 8th node (both components) plus the
full vector's 2-norm for the 2M-DOF plate (the full vector is 16 MB).

It also times short bounded solves (the number of iterations the benchmark's CPU sample runs)
on the same system, so the per-iteration cost of the sample can be checked against the full run.

Run where the reference core has been built (`make -C oracle ref`); it takes about half an
hour on one core:

    python tests/golden/make_golden_large.py [--only 400x1250|565x1766]
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import RefCore, build  # noqa: E402

plate = importlib.import_module("mpi-cst-fem-solver_b200.plate")

PLATES = {"400x1250": (400, 1250, "full"), "565x1766": (565, 1766, "sub8")}
SAMPLE_ITERS = 50
SUB_STRIDE = 8


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def run_plate(R: RefCore, n_r: int, n_theta: int, store: str) -> None:
    tag = f"{n_r}x{n_theta}"
    timing = {}
    t = time.perf_counter()
    p = plate.quarter_plate(n_r, n_theta)
    m = R.mesh_from_arrays(p.xy, p.triangles, p.boundary_edges)
    D = R.constitutive_matrix(1.0, 0.3, 0)
    t0 = time.perf_counter()
    K = R.pattern(m)
    t1 = time.perf_counter()
    R.assemble(m, D, 1.0, K)
    t2 = time.perf_counter()
    f = np.zeros(p.num_dofs)
    R.add_traction(m, "right", 1.0, 1.0, 0.0, f)
    t3 = time.perf_counter()
    f0 = f.copy()
    rp, cols, kv = R.csr_arrays(K)
    dofs, vals = R.dirichlet_dofs(m, [("left_sym", 0, 0.0), ("bottom_sym", 1, 0.0)])
    t4 = time.perf_counter()
    R.apply_dirichlet(K, dofs, vals, f)
    t5 = time.perf_counter()
    timing.update(build_stiffness_pattern_s=t1 - t0, assemble_stiffness_s=t2 - t1,
                  add_traction_s=t3 - t2, apply_dirichlet_s=t5 - t4)
    _, _, kbc = R.csr_arrays(K)
    print(f"[{tag}] setup done in {time.perf_counter() - t:.1f} s; solving", flush=True)
    x, st = R.pcg(K, f, 1e-10, 400000, record_history=True)
    timing.update(solver_setup_s=st["t_setup"], solve_s=st["t_solve"], spmv_s=st["t_spmv"],
                  dot_s=st["t_dot"], vector_ops_s=st["t_vec"])
    per_it = st["t_solve"] / max(st["iterations"], 1)
    print(f"[{tag}] {st['iterations']} iterations in {st['t_solve']:.1f} s "
          f"({per_it * 1e3:.2f} ms/it), true {st['true_rel_residual']:.3e}", flush=True)
    samples = []
    for _ in range(3):
        _, s2 = R.pcg(K, f, 1e-30, SAMPLE_ITERS)
        samples.append(s2["t_solve"] / SAMPLE_ITERS)
    es = R.element_stresses(m, x, 1.0, 0.3, 0)
    e = int(np.argmin(np.hypot(es["cx"], es["cy"] - 1.0)))
    hist = st["residual_history"]
    meta = {
        "n_r": n_r, "n_theta": n_theta, "n_dofs": int(p.num_dofs), "nnz": int(cols.size),
        "xy_sha": sha(p.xy), "tri_sha": sha(p.triangles),
        "row_ptr_sha": sha(rp), "cols_sha": sha(cols), "K_sha": sha(kv), "Kbc_sha": sha(kbc),
        "f_sha": sha(f0), "b_sha": sha(f), "dir_dofs_sha": sha(dofs),
        "iters": int(st["iterations"]), "converged": bool(st["converged"]),
        "rel": float(st["rel_residual"]), "true_rel": float(st["true_rel_residual"]),
        "message": st["message"], "warning": st["warning"],
        "u_sha": sha(x), "u_norm": float(np.linalg.norm(x)), "b_norm": float(np.linalg.norm(f)),
        "scf": float(es["sxx"][e]), "scf_element": e,
        "sxx_sha": sha(es["sxx"]),
        "hist_every_1000": [float(v) for v in hist[::1000]],
        "u_store": store, "u_stride_nodes": SUB_STRIDE if store == "sub8" else 1,
        "cpu_run": {
            "what": "reference serial core (oracle/_ref, compiled from the reference's src/*.cpp "
                    "with g++ -O3), one process, one thread",
            "cores_used": 1, "nproc": os.cpu_count(), "cpu_model": cpu_model(),
            "date": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            **{k: round(v, 4) for k, v in timing.items()},
            "per_iter_full_s": per_it,
            "sample_iters": SAMPLE_ITERS,
            "per_iter_sample_s": samples,
            "sample_vs_full": [s / per_it for s in samples],
        },
    }
    if store == "full":
        np.savez_compressed(os.path.join(HERE, f"plate_{tag}.npz"), u=x)
    else:
        nodes = np.arange(0, p.num_nodes, SUB_STRIDE)
        idx = np.stack([2 * nodes, 2 * nodes + 1], axis=1).reshape(-1)
        np.savez_compressed(os.path.join(HERE, f"plate_{tag}.npz"), u_sub=x[idx])
    with open(os.path.join(HERE, f"plate_{tag}.json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    R.free_csr(K)
    R.free_mesh(m)
    print(f"[{tag}] written", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=sorted(PLATES))
    a = ap.parse_args()
    build(ref=True)
    R = RefCore()
    for tag, (n_r, n_theta, store) in PLATES.items():
        if a.only and tag != a.only:
            continue
        run_plate(R, n_r, n_theta, store)


if __name__ == "__main__":
    main()
