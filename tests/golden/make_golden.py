"""Generates the golden fixtures of this directory from the reference's own serial core.

Run where the reference sources exist (they are compiled by `make -C oracle ref` into
oracle/_ref/libcstfem_ref.so; this script reads the reference checkout, by default the
directory `reference` beside this repository or $CSTFEM_REF, for its two committed Kirsch meshes):

    python tests/golden/make_golden.py [--ref PATH]

Every number stored here was computed by the reference's code (read_gmsh, cst_stiffness,
build_stiffness_pattern, assemble_stiffness, add_traction, add_dirichlet, apply_dirichlet,
CgJacobiSolver); the tests compare the oracle restatement and the GPU path against them.
Large arrays are stored as SHA-256 digests of their bytes.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import REF_DIR, RefCore, build  # noqa: E402

plate = importlib.import_module("mpi-cst-fem-solver_b200.plate")
GROUPS = ("hole", "left_sym", "bottom_sym", "right", "top")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def kirsch_case(R: RefCore, path: str, out: str, full: bool):
    """Reference pipeline on a Kirsch mesh: E=210e9, nu=0.3, t=0.01, symmetry BCs,
    traction (100e6, 0) on `right`, rtol 1e-10 and 1e-12, plane stress and strain."""
    m = R.read_gmsh(path)
    xy, tri, groups, flipped = R.mesh_arrays(m, GROUPS)
    rec = {"xy": xy, "tri": tri, "flipped": np.array(flipped)}
    for g, e in groups.items():
        rec["group_" + g] = e
    dofs, vals = R.dirichlet_dofs(m, [("left_sym", 0, 0.0), ("bottom_sym", 1, 0.0)])
    rec["dir_dofs"], rec["dir_vals"] = dofs, vals
    meta = {}
    for plane in (0, 1):
        tag = "strain" if plane else "stress"
        D = R.constitutive_matrix(210e9, 0.3, plane)
        K = R.pattern(m)
        R.assemble(m, D, 0.01, K)
        rp, cols, kv = R.csr_arrays(K)
        f = np.zeros(xy.size)
        R.add_traction(m, "right", 0.01, 100e6, 0.0, f)
        rec[f"{tag}_f"] = f.copy()
        R.apply_dirichlet(K, dofs, vals, f)
        _, _, kbc = R.csr_arrays(K)
        if full:
            rec["row_ptr"], rec["cols"] = rp, cols
            rec[f"{tag}_K"], rec[f"{tag}_Kbc"] = kv, kbc
        meta[f"{tag}_K_sha"], meta[f"{tag}_Kbc_sha"] = sha(kv), sha(kbc)
        meta["row_ptr_sha"], meta["cols_sha"], meta["nnz"] = sha(rp), sha(cols), int(cols.size)
        rec[f"{tag}_b"] = f
        for rtol, rt in ((1e-10, "10"), (1e-12, "12")):
            x, st = R.pcg(K, f, rtol, 20000, record_history=True)
            rec[f"{tag}_u{rt}"] = x
            rec[f"{tag}_hist{rt}"] = st["residual_history"]
            meta[f"{tag}_iters{rt}"] = st["iterations"]
            meta[f"{tag}_true{rt}"] = st["true_rel_residual"]
            meta[f"{tag}_msg{rt}"] = st["message"]
        es = R.element_stresses(m, rec[f"{tag}_u10"], 210e9, 0.3, plane)
        for k in ("sxx", "syy", "txy", "von_mises", "szz", "cx", "cy", "area"):
            meta[f"{tag}_stress_{k}_sha"] = sha(es[k])
        rec[f"{tag}_sxx"] = es["sxx"]
        R.free_csr(K)
    R.free_mesh(m)
    np.savez_compressed(out + ".npz", **rec)
    with open(out + ".json", "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)


def plate_case(R: RefCore, n_r: int, n_theta: int, out: str):
    """The 40 x 80 O-grid plate (E=1, nu=0.3, plane stress, t=1, traction (1,0) on right)."""
    p = plate.quarter_plate(n_r, n_theta)
    m = R.mesh_from_arrays(p.xy, p.triangles, p.boundary_edges)
    D = R.constitutive_matrix(1.0, 0.3, 0)
    K = R.pattern(m)
    R.assemble(m, D, 1.0, K)
    rp, cols, kv = R.csr_arrays(K)
    f = np.zeros(p.num_dofs)
    R.add_traction(m, "right", 1.0, 1.0, 0.0, f)
    f0 = f.copy()
    dofs, vals = R.dirichlet_dofs(m, [("left_sym", 0, 0.0), ("bottom_sym", 1, 0.0)])
    R.apply_dirichlet(K, dofs, vals, f)
    _, _, kbc = R.csr_arrays(K)
    x, st = R.pcg(K, f, 1e-10, 20000, record_history=True)
    es = R.element_stresses(m, x, 1.0, 0.3, 0)
    d = np.hypot(es["cx"], es["cy"] - 1.0)
    e = int(np.argmin(d))
    meta = {"n_r": n_r, "n_theta": n_theta, "xy_sha": sha(p.xy), "tri_sha": sha(p.triangles),
            "row_ptr_sha": sha(rp), "cols_sha": sha(cols), "K_sha": sha(kv), "Kbc_sha": sha(kbc),
            "f_sha": sha(f0), "b_sha": sha(f), "iters": st["iterations"],
            "true_rel": st["true_rel_residual"], "rel": st["rel_residual"], "nnz": int(cols.size),
            "scf": float(es["sxx"][e]), "scf_element": e}
    np.savez_compressed(out + ".npz", b=f, u=x, hist=st["residual_history"], dir_dofs=dofs)
    with open(out + ".json", "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    R.free_csr(K)
    R.free_mesh(m)


def element_case(R: RefCore, out: str):
    """Ke of random counter-clockwise triangles (seeded), both plane conditions."""
    rng = np.random.default_rng(12345)
    tris = []
    while len(tris) < 20:
        xy = rng.uniform(-2.0, 3.0, 6)
        A = 0.5 * ((xy[2] - xy[0]) * (xy[5] - xy[1]) - (xy[4] - xy[0]) * (xy[3] - xy[1]))
        if abs(A) < 0.5:
            continue
        if A < 0:
            xy[[2, 3, 4, 5]] = xy[[4, 5, 2, 3]]
        tris.append(xy)
    tris = np.array(tris)
    rec = {"xy": tris}
    for plane in (0, 1):
        D = R.constitutive_matrix(210e9, 0.3, plane)
        rec[f"D{plane}"] = D
        rec[f"K{plane}"] = np.array([R.cst_stiffness(t, D, 0.01) for t in tris])
    np.savez_compressed(out + ".npz", **rec)


def spd_case(R: RefCore, out: str):
    """Random SPD D A D systems (the reference's test_pcg.cpp construction, numpy-seeded),
    solved by the reference's CgJacobiSolver at rtol 1e-12."""
    rng = np.random.default_rng(2026)
    rec = {}
    for n in (5, 40, 120):
        M = rng.uniform(-1.0, 1.0, (n, n))
        A = M.T @ M + n * np.eye(n)
        d = 10.0 ** (3.0 * (rng.uniform(-1.0, 1.0, n) + 1.0) / 2.0)
        A = A * d[:, None] * d[None, :]
        b = rng.uniform(-1.0, 1.0, n)
        rp = np.arange(0, n * n + 1, n, dtype=np.int32)
        cols = np.tile(np.arange(n, dtype=np.int32), n)
        K = R.csr(n, rp, cols, A.reshape(-1))
        x, st = R.pcg(K, b, 1e-12, 1000, record_history=True)
        rec[f"A{n}"], rec[f"b{n}"], rec[f"x{n}"] = A, b, x
        rec[f"iters{n}"] = np.array(st["iterations"])
        R.free_csr(K)
    np.savez_compressed(out + ".npz", **rec)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=REF_DIR)
    a = ap.parse_args()
    build(ref=True)
    R = RefCore()
    data = os.path.join(a.ref, "tests", "data")
    kirsch_case(R, os.path.join(data, "kirsch_L0.msh"), os.path.join(HERE, "kirsch_L0"), full=True)
    kirsch_case(R, os.path.join(data, "kirsch_L1.msh"), os.path.join(HERE, "kirsch_L1"), full=False)
    plate_case(R, 40, 80, os.path.join(HERE, "plate_40x80"))
    element_case(R, os.path.join(HERE, "element"))
    spd_case(R, os.path.join(HERE, "spd"))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
