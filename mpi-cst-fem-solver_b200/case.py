"""Case-file front end: runs a reference case file (src/case.cpp, src/driver.cpp:34-90,164-298)
on the GPU path.

    python -m mpi-cst-fem-solver_b200.case cases/kirsch_L0.case

The file format and keys are the reference's (`key = value`, `#` comments, duplicate keys and
keys with whitespace rejected, unknown keys warned about). `solver` selects the GPU method:
`cg_jacobi` (the reference's recurrence and stopping rule, FP64), `gpu_cg` (FP64, stop on the
FP64 true residual), `gpu_cg_mixed` (FP32 operator, FP64 vectors), `gpu_cg_learned` (the learned
preconditioner in flexible CG) or `gpu_cg_amg` (smoothed-aggregation multigrid V-cycle in flexible
CG); `petsc` and `path = distributed` are not available on this path.
Outputs in `output_dir`: timings.json (the reference's layout, "path": "gpu"), displacement.npy
(2 per node) and element_stresses.npz; Kirsch cases also report the stress concentration factor
and the relative L2 error of the centroid stresses against the analytical field. VTU output is
not written (out of scope). Exit code: 0 converged, 2 not converged, 1 error.
"""
from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np

from .mesh_io import read_gmsh
from .native import CstgError
from .solver import (CgJacobiSolver, DirichletDofs, PlaneCondition, SolverOptions, add_dirichlet_group,
                     add_kirsch_traction, add_traction, apply_dirichlet, assemble_stiffness,
                     build_stiffness_pattern, compute_element_stresses, constitutive_matrix, scf_at_hole)

KNOWN_KEYS = ["mesh", "plane", "E", "nu", "thickness", "partitioner", "solver", "rtol", "max_iter", "output_dir",
              "bc.dirichlet", "bc.traction", "kirsch.sigma_inf", "kirsch.a", "path", "instrument",
              "petsc.near_nullspace", "petsc.options", "petsc.log_view"]
SOLVERS = {"cg_jacobi": dict(precision="fp64", true_residual_stop=False),
           "gpu_cg": dict(precision="fp64", true_residual_stop=True),
           "gpu_cg_mixed": dict(precision="mixed", true_residual_stop=True),
           "gpu_cg_learned": dict(precision="mixed", true_residual_stop=True, preconditioner="learned_mg"),
           "gpu_cg_learned_local": dict(precision="mixed", true_residual_stop=True, preconditioner="learned"),
           "gpu_cg_amg": dict(precision="fp64", true_residual_stop=True, preconditioner="amg")}


class CaseError(RuntimeError):
    pass


class CaseFile:
    """`key = value` entries with their line numbers (case.cpp:25-58)."""

    def __init__(self, source: str):
        self.source = source
        self.entries = {}
        self.order = []

    @classmethod
    def load(cls, path: str) -> "CaseFile":
        try:
            text = open(path).read()
        except OSError:
            raise CaseError(f"{path}: cannot open file")
        return cls.parse(text, path)

    @classmethod
    def parse(cls, text: str, source: str = "<case>") -> "CaseFile":
        cf = cls(source)
        for no, raw in enumerate(text.splitlines(), start=1):
            line = raw.split("#", 1)[0].strip(" \t\r")
            if not line:
                continue
            if "=" not in line:
                raise CaseError(f"{source}:{no}: expected 'key = value', got '{line}'")
            key, value = (s.strip(" \t\r") for s in line.split("=", 1))
            if not key:
                raise CaseError(f"{source}:{no}: empty key")
            if any(c in key for c in " \t"):
                raise CaseError(f"{source}:{no}: key '{key}' contains whitespace")
            if key in cf.entries:
                raise CaseError(f"{source}:{no}: duplicate key '{key}' (first defined on line "
                                f"{cf.entries[key][1]})")
            cf.entries[key] = (value, no)
            cf.order.append(key)
        return cf

    def has(self, key):
        return key in self.entries

    def get_string(self, key, fallback=None):
        if key not in self.entries:
            if fallback is None:
                raise CaseError(f"{self.source}: missing required key '{key}'")
            return fallback
        return self.entries[key][0]

    def get_double(self, key, fallback=None):
        if key not in self.entries and fallback is not None:
            return float(fallback)
        v = self.get_string(key)
        try:
            x = float(v)
        except ValueError:
            raise CaseError(f"{self.source}:{self.entries[key][1]}: key '{key}': '{v}' is not a number")
        if not math.isfinite(x):
            raise CaseError(f"{self.source}:{self.entries[key][1]}: key '{key}': '{v}' is not a number")
        return x

    def get_int(self, key, fallback=None):
        if key not in self.entries and fallback is not None:
            return int(fallback)
        v = self.get_string(key)
        try:
            return int(v, 10)
        except ValueError:
            raise CaseError(f"{self.source}:{self.entries[key][1]}: key '{key}': '{v}' is not an integer")

    def warn_unknown_keys(self, known, err) -> int:
        unknown = [k for k in self.order if k not in known]
        for k in unknown:
            err.write(f"warning: {self.source}:{self.entries[k][1]}: unknown key '{k}'\n")
        return len(unknown)


def parse_group_list(text: str, what: str):
    """'group:key=val,key=val ; group:key=val' (bc.cpp:38-64)."""
    out = []
    for item in (s.strip(" \t") for s in text.split(";")):
        if not item:
            continue
        if ":" not in item:
            raise CaseError(f"{what}: expected 'group:key=value' in '{item}'")
        group, rest = item.split(":", 1)
        group = group.strip(" \t")
        if not group:
            raise CaseError(f"{what}: empty group in '{item}'")
        kv = []
        for assign in (s.strip(" \t") for s in rest.split(",")):
            if "=" not in assign:
                raise CaseError(f"{what}: expected 'key=value' in '{item}'")
            k, v = (s.strip(" \t") for s in assign.split("=", 1))
            try:
                x = float(v)
                if not math.isfinite(x):
                    raise ValueError
            except ValueError:
                raise CaseError(f"{what} '{group}:{k}': '{v}' is not a number")
            kv.append((k, x))
        if not kv:
            raise CaseError(f"{what}: no values for '{group}'")
        out.append((group, kv))
    return out


def parse_dirichlet(text: str):
    specs = []
    for group, kv in parse_group_list(text, "bc.dirichlet"):
        s = {"group": group}
        for k, v in kv:
            if k not in ("ux", "uy"):
                raise CaseError(f"bc.dirichlet: unknown component '{k}' for group '{group}' (use ux or uy)")
            if k in s:
                raise CaseError(f"bc.dirichlet: '{k}' given twice for group '{group}'")
            s[k] = v
        specs.append(s)
    return specs


def parse_traction(text: str):
    specs = []
    for group, kv in parse_group_list(text, "bc.traction"):
        s = {"group": group, "tx": 0.0, "ty": 0.0}
        seen = set()
        for k, v in kv:
            if k not in ("tx", "ty"):
                raise CaseError(f"bc.traction: unknown component '{k}' for group '{group}' (use tx or ty)")
            if k in seen:
                raise CaseError(f"bc.traction: '{k}' given twice for group '{group}'")
            seen.add(k)
            s[k] = v
        specs.append(s)
    return specs


def read_case_settings(c: CaseFile) -> dict:
    s = {"mesh": c.get_string("mesh"), "output_dir": c.get_string("output_dir", "results"),
         "plane_name": c.get_string("plane")}
    if s["plane_name"] not in ("plane_stress", "plane_strain"):
        raise CaseError(f"{c.source}: plane must be plane_stress or plane_strain, got '{s['plane_name']}'")
    s["plane"] = PlaneCondition.Stress if s["plane_name"] == "plane_stress" else PlaneCondition.Strain
    s["E"], s["nu"], s["thickness"] = c.get_double("E"), c.get_double("nu"), c.get_double("thickness")
    if not s["E"] > 0:
        raise CaseError(f"{c.source}: E must be positive")
    if not -1.0 < s["nu"] < 0.5:
        raise CaseError(f"{c.source}: nu must be in (-1, 0.5)")
    if not s["thickness"] > 0:
        raise CaseError(f"{c.source}: thickness must be positive")
    part = c.get_string("partitioner", "metis")
    if part not in ("metis", "parmetis"):
        raise CaseError(f"{c.source}: partitioner must be metis or parmetis")
    inst = c.get_string("instrument", "true")
    if inst not in ("true", "false"):
        raise CaseError(f"{c.source}: instrument must be true or false")
    s["instrument"] = inst == "true"
    path = c.get_string("path", "auto")
    if path not in ("auto", "serial", "distributed"):
        raise CaseError(f"{c.source}: path must be auto, serial or distributed, got '{path}'")
    if path == "distributed":
        raise CaseError(f"{c.source}: path = distributed is not available on the GPU path (one device-resident "
                        "matrix); use path = auto or serial")
    solver = c.get_string("solver", "cg_jacobi")
    if solver == "petsc":
        raise CaseError(f"{c.source}: solver = petsc is not available on the GPU path")
    if solver not in SOLVERS:
        raise CaseError(f"{c.source}: solver must be one of {', '.join(SOLVERS)}, got '{solver}'")
    s["solver"] = solver
    s["rtol"] = c.get_double("rtol", 1e-10)
    s["max_iter"] = c.get_int("max_iter", 20000)
    return s


def _kirsch_stress(a, s_inf, x, y):
    """Analytical Kirsch stresses at points (kirsch.cpp:7-38)."""
    r, th = np.hypot(x, y), np.arctan2(y, x)
    q2 = a * a / (r * r)
    q4 = q2 * q2
    c2, s2 = np.cos(2 * th), np.sin(2 * th)
    rr = 0.5 * s_inf * (1 - q2) + 0.5 * s_inf * (1 - 4 * q2 + 3 * q4) * c2
    tt = 0.5 * s_inf * (1 + q2) - 0.5 * s_inf * (1 + 3 * q4) * c2
    rt = -0.5 * s_inf * (1 + 2 * q2 - 3 * q4) * s2
    c, n = np.cos(th), np.sin(th)
    return (rr * c * c + tt * n * n - 2 * rt * n * c, rr * n * n + tt * c * c + 2 * rt * n * c,
            (rr - tt) * n * c + rt * (c * c - n * n))


def run_case(case_path: str, out=sys.stdout, err=sys.stderr, device: int = 0) -> int:
    try:
        import torch
        t_total = time.perf_counter()
        t0 = time.perf_counter()
        c = CaseFile.load(case_path)
        c.warn_unknown_keys(KNOWN_KEYS, err)
        s = read_case_settings(c)
        mesh = read_gmsh(s["mesh"])
        t_read = time.perf_counter() - t0
        out.write(f"mesh {s['mesh']}: {mesh.num_nodes} nodes, {mesh.num_triangles} triangles, "
                  f"{mesh.num_dofs} DOFs\n")

        t0 = time.perf_counter()
        D = constitutive_matrix(s["E"], s["nu"], s["plane"])
        K = build_stiffness_pattern(mesh)
        assemble_stiffness(mesh, D, s["thickness"], K)
        torch.cuda.synchronize(device)
        t_asm = time.perf_counter() - t0

        t0 = time.perf_counter()
        f = torch.zeros(mesh.num_dofs, dtype=torch.float64, device=device)
        spec = c.get_string("bc.traction", "")
        kirsch = None
        if spec == "kirsch_exact":
            kirsch = (c.get_double("kirsch.sigma_inf"), c.get_double("kirsch.a"))
            if not kirsch[1] > 0:
                raise CaseError(f"{c.source}: kirsch.a must be positive")
            for grp in ("right", "top"):
                if grp not in mesh.boundary_edges:
                    raise CaseError(f"unknown boundary group '{grp}'")
                add_kirsch_traction(K, mesh.boundary_edges[grp], s["thickness"], kirsch[1], kirsch[0], f)
        else:
            for tr in parse_traction(spec):
                if tr["group"] not in mesh.boundary_edges:
                    raise CaseError(f"unknown boundary group '{tr['group']}'")
                add_traction(K, mesh.boundary_edges[tr["group"]], s["thickness"], tr["tx"], tr["ty"], f)
        dofs = DirichletDofs()
        for d in parse_dirichlet(c.get_string("bc.dirichlet", "")):
            if "ux" in d:
                add_dirichlet_group(mesh, d["group"], 0, d["ux"], dofs)
            if "uy" in d:
                add_dirichlet_group(mesh, d["group"], 1, d["uy"], dofs)
        apply_dirichlet(dofs, K, f)
        torch.cuda.synchronize(device)
        t_bcs = time.perf_counter() - t0

        t0 = time.perf_counter()
        # cg_jacobi with instrument = true: the phases timed with CUDA events (SolveBreakdown)
        instrumented = s["solver"] == "cg_jacobi" and s.get("instrument", False)
        opts = SolverOptions(rtol=s["rtol"], max_iter=s["max_iter"], **SOLVERS[s["solver"]],
                             **({"launch": "instrumented"} if instrumented else {}))
        solver = CgJacobiSolver(opts)
        solver.setup(K)
        if opts.preconditioner in ("learned", "learned_mg"):
            from . import learned
            mode = "cycle" if opts.preconditioner == "learned_mg" else "local"
            learned.setup(K, learned.load_weights(mode=mode), learned.node_material(D, mesh.num_nodes))
        u_d = torch.zeros_like(f)
        st = solver.solve(f, u_d)
        u = u_d.cpu().numpy()
        t_solve = time.perf_counter() - t0
        out.write(f"{s['solver']}: {st.message}; true relative residual {st.true_rel_residual}\n")
        if st.warning:
            err.write(st.warning + "\n")
        if not st.converged:
            err.write(f"error: solver did not converge: {st.message}\n")

        t0 = time.perf_counter()
        os.makedirs(s["output_dir"], exist_ok=True)
        es = compute_element_stresses(K, u, s["E"], s["nu"], s["plane"])
        np.save(os.path.join(s["output_dir"], "displacement.npy"), u)
        np.savez(os.path.join(s["output_dir"], "element_stresses.npz"), **es)
        kj = None
        if kirsch:
            scf, e = scf_at_hole(es, kirsch[1], kirsch[0])
            sxx, syy, txy = _kirsch_stress(kirsch[1], kirsch[0], es["cx"], es["cy"])
            num = np.sum(es["area"] * ((es["sxx"] - sxx) ** 2 + (es["syy"] - syy) ** 2 + 2 * (es["txy"] - txy) ** 2))
            den = np.sum(es["area"] * (sxx ** 2 + syy ** 2 + 2 * txy ** 2))
            ana = _kirsch_stress(kirsch[1], kirsch[0], es["cx"][e], es["cy"][e])[0] / kirsch[0]
            kj = {"sigma_inf": kirsch[0], "a": kirsch[1], "l2_rel_stress_error": float(np.sqrt(num / den)),
                  "scf": {"element": e, "x": float(es["cx"][e]), "y": float(es["cy"][e]), "numerical": float(scf),
                          "analytical_at_centroid": float(ana), "theoretical": 3.0}}
            out.write(f"Kirsch: relative L2 error of the centroid stresses {kj['l2_rel_stress_error']}; SCF at "
                      f"centroid ({kj['scf']['x']}, {kj['scf']['y']}): numerical {scf}, analytical {ana}, "
                      f"theoretical 3\n")
        t_out = time.perf_counter() - t0
        t_all = time.perf_counter() - t_total
        timings = {
            "case": case_path, "mesh": s["mesh"], "ranks": 1, "path": "gpu",
            "device": torch.cuda.get_device_name(device), "plane": s["plane_name"], "nodes": mesh.num_nodes,
            "elements": mesh.num_triangles, "dofs": mesh.num_dofs, "nnz": K.nnz(),
            "solver": {"name": s["solver"], "rtol": s["rtol"], "max_iter": s["max_iter"],
                       "iterations": st.iterations, "rel_residual": st.rel_residual,
                       "true_rel_residual": st.true_rel_residual, "converged": st.converged,
                       "device_solve_seconds": st.solve_seconds},
            "solve_breakdown": _breakdown_json(solver.breakdown(), st.iterations) if instrumented else None,
            "timings": {"read": t_read, "assembly": t_asm, "bcs": t_bcs, "solve": t_solve, "output": t_out,
                        "total": t_all},
            "kirsch": kj}
        with open(os.path.join(s["output_dir"], "timings.json"), "w") as js:
            json.dump(timings, js, indent=2)
        out.write(f"wrote {os.path.join(s['output_dir'], 'timings.json')}, displacement.npy, element_stresses.npz\n"
                  f"time: read {t_read} s, assembly {t_asm} s, bcs {t_bcs} s, solve {t_solve} s, output {t_out} s, "
                  f"total {t_all} s\n")
        K.ctx.close()
        return 0 if st.converged else 2
    except (CaseError, CstgError, OSError) as e:
        err.write(f"error: {e}\n")
        return 1


def _breakdown_json(bd: dict, iterations: int) -> dict:
    """The reference's solve_breakdown entries (driver.cpp:92-110, one rank: min = max = mean) from
    the device phase times of an instrumented solve; the halo and allreduce phases of the
    distributed path have no counterpart on one device and are 0."""
    acc = bd["setup"] + bd["spmv_local"] + bd["dot_local"] + bd["vector_ops"]
    vals = [("setup", bd["setup"]), ("spmv_local", bd["spmv_local"]), ("halo_post", 0.0), ("halo_wait", 0.0),
            ("spmv_ghost", 0.0), ("dot_local", bd["dot_local"]), ("allreduce", 0.0),
            ("vector_ops", bd["vector_ops"]), ("unaccounted", bd["total"] - acc), ("total", bd["total"]),
            ("time_per_iteration", bd["total"] / iterations if iterations > 0 else 0.0),
            ("accounted_fraction", acc / bd["total"] if bd["total"] > 0 else 0.0),
            ("halo_bytes_sent_per_iteration", 0.0), ("halo_messages_sent_per_iteration", 0.0)]
    return {k: {"min": v, "max": v, "mean": v} for k, v in vals}


def main():
    if len(sys.argv) != 2:
        sys.stderr.write("usage: python -m mpi-cst-fem-solver_b200.case <file.case>\n")
        return 1
    return run_case(sys.argv[1])


if __name__ == "__main__":
    sys.exit(main())
