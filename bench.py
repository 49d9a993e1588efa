#!/usr/bin/env python
"""Time-to-solve benchmark of the CST assembly -> loads -> Dirichlet -> preconditioned CG path on B200.

A step is one full pass of the path over one synthetic plate: stiffness pattern, assembly,
traction loads (on the GPU), Dirichlet elimination, Jacobi setup, preconditioner setup and
flexible CG to rtol 1e-10 on the FP64 TRUE residual (||b - A x|| / ||b||). The default workload
is the 2M-DOF quarter plate (O-grid n_r = 565 x n_theta = 1766, 2,000,244 DOFs, 27,966,096
nonzeros; E = 1, nu = 0.3, plane stress, t = 1, traction (1, 0) on x = 10, u_x = 0 on x = 0,
u_y = 0 on y = 0).

The timed solve is the learned preconditioner in mixed precision: the multigrid cycle whose
finest-level post-smoother is the trained message-passing network (BF16 tensor-core layers),
FP32 cycle operators and SpMV, FP64 vectors, scalars and reliable updates, inside flexible CG.
Beside it, on the same matrix: plain FP64 Jacobi-PCG on the GPU (the method the learned solve is
compared with), mixed Jacobi-PCG, the Chebyshev multigrid cycle without a network, the same
learned cycle with the network at zero, and each solution's error against the reference
serial core's displacements (tests/golden, computed by the reference's own code).

  value  DOFs solved per second with the mesh, loads and BCs already in HBM (CUDA events on
         the work stream), summed over all GPUs (independent replicas, weak scaling).
  e2e    the same through the C ABI with pinned HOST buffers: every step uploads the mesh,
         edges and BCs and downloads the displacements (wall clock around the step).

One JSON line on rank 0. `--impl reference` times the reference's own CPU path (compiled from
its sources into oracle/_ref) on this host's cores instead, on bounded samples of its solve,
next to the committed record of its full run.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    # name: (n_r, n_theta, description)
    "plate2m": (565, 1766, "quarter plate [0,10]^2 minus r<1, O-grid n_r=565 x n_theta=1766"),
    "plate1m": (400, 1250, "quarter plate [0,10]^2 minus r<1, O-grid n_r=400 x n_theta=1250"),
    "plate4m": (800, 2500, "quarter plate [0,10]^2 minus r<1, O-grid n_r=800 x n_theta=2500"),
    "plate8m": (1131, 3536, "quarter plate [0,10]^2 minus r<1, O-grid n_r=1131 x n_theta=3536"),
    "plate40x80": (40, 80, "quarter plate [0,10]^2 minus r<1, O-grid n_r=40 x n_theta=80"),
}

# Committed records of the reference serial core run to convergence on the build host
# (tests/golden/make_golden_large.py): iterations, wall seconds per phase, host.
GOLDEN = os.path.join(REPO, "tests", "golden")
RECORDS = {"plate2m": "plate_565x1766", "plate1m": "plate_400x1250", "plate40x80": "plate_40x80"}

METRIC = ("time-to-solve @rtol 1e-10 (FP64 true residual), 2M-DOF plate, learned preconditioner + mixed "
          "precision, as DOFs solved per second")

PRECONDS = {"learned": "learned_mg", "learned_local": "learned", "amg": "amg", "jacobi": "jacobi"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plate2m", choices=sorted(WORKLOADS))
    ap.add_argument("--precond", default="learned", choices=sorted(PRECONDS),
                    help="preconditioner of the timed solve: the learned multigrid cycle (default: the "
                         "trained network as the cycle's post-smoother), the network alone "
                         "(learned_local), the Chebyshev multigrid cycle (amg) or Jacobi")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-sample-iters", type=int, default=150)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the comparison solves")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-solve measurement")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the large plate (n_r=800 x n_theta=2500): learned + mixed against plain FP64")
    ap.add_argument("--only", choices=["spmv", "solve", "batch", "learned", "network", "amg"], default=None,
                    help="profiling modes (one JSON line each): `spmv` --reps SpMV launches, `solve` one "
                         "full step, `batch` the 64-plate x 4-load-case batched solve, `learned` the "
                         "network's stages after a step, `network` the network's stages on the assembled "
                         "system without a solve, `amg` the multigrid cycle")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--max-iter", type=int, default=200000,
                    help="iteration cap of the solves (profiling captures use a small cap)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    return a


# ---- distributed plumbing (replicas: barrier + max over ranks only) -------------------------

class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str):
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float, device=None) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def timed_region(step, k: int, w: int, dist: Dist, start_timer, stop_timer, sync) -> float:
    """W untimed steps, then K steps bracketed by barrier + sync on both sides; returns the
    max over ranks of the elapsed seconds (the timer pair may be CUDA events or a clock)."""
    for _ in range(w):
        step()
    sync()
    dist.barrier()
    sync()
    t = start_timer()
    for _ in range(k):
        step()
    el = stop_timer(t)
    sync()
    dist.barrier()
    return el


# ---- clocks -----------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        return parse_clock_csv(out)


def parse_clock_csv(text: str) -> dict:
    """Median SM clock, max clock and the throttle reasons seen (ClockSampler.FIELDS order)."""
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in text.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 7:
            continue
        try:
            sm.append(float(f[0]))
            mx = float(f[1])
        except ValueError:
            continue
        for name, v in zip(names, f[3:7]):
            if v.lower().startswith("active"):
                reasons.add(name)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


# ---- helpers ------------------------------------------------------------------------------------

def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name: str, key: str = "dram_bytes_per_launch_full_size"):
    """A DRAM byte count (per launch, or per PCG iteration) from a committed ncu summary, if present."""
    p = os.path.join(REPO, "profiles", name)
    if not os.path.exists(p):
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def make_inputs(pkg, workload):
    n_r, n_t, _ = WORKLOADS[workload]
    mesh = pkg.plate.quarter_plate(n_r, n_t)
    D = pkg.constitutive_matrix(1.0, 0.3)
    dofs, vals = pkg.plate.symmetry_dirichlet(mesh)
    return mesh, D, dofs, vals


def reference_record(workload):
    """The reference serial core's full run on this workload (tests/golden/plate_*.json/.npz):
    its iterations, true residual, SCF, displacements (all or a subsample) and wall-clock record."""
    name = RECORDS.get(workload)
    if not name or not os.path.exists(os.path.join(GOLDEN, name + ".json")):
        return None
    meta = json.load(open(os.path.join(GOLDEN, name + ".json")))
    npz = np.load(os.path.join(GOLDEN, name + ".npz"))
    if "u_sub" in npz.files:
        stride = int(meta.get("u_stride_nodes", 8))
        n_nodes = meta["n_dofs"] // 2
        nodes = np.arange(0, n_nodes, stride)
        idx = np.stack([2 * nodes, 2 * nodes + 1], axis=1).reshape(-1)
        u = npz["u_sub"]
    else:
        idx, u = None, npz["u"]
    return {"meta": meta, "u": u, "idx": idx, "file": f"tests/golden/{name}.json"}


def rel_error_vs_reference(rec, x):
    """||x - u_ref|| / ||u_ref|| over the DOFs the record holds (all, or every 8th node)."""
    if rec is None:
        return None
    xs = x if rec["idx"] is None else x[rec["idx"]]
    return float(np.linalg.norm(xs - rec["u"]) / np.linalg.norm(rec["u"]))


# ---- CPU baseline: the reference's serial core on a bounded sample ---------------------------------

def cpu_sample(mesh, dofs, vals, sample_iters: int):
    """Times the reference's CPU path (oracle/_ref) on this plate: full pattern + assembly +
    loads + BCs, then `sample_iters` PCG iterations. Falls back to the oracle restatement."""
    import oracle
    if oracle.RefCore.available():
        R = oracle.RefCore()
        t0 = time.perf_counter()
        m = R.mesh_from_arrays(mesh.xy, mesh.triangles, mesh.boundary_edges)
        K = R.pattern(m)
        R.assemble(m, R.constitutive_matrix(1.0, 0.3), 1.0, K)
        f = np.zeros(mesh.num_dofs)
        R.add_traction(m, "right", 1.0, 1.0, 0.0, f)
        R.apply_dirichlet(K, dofs, vals, f)
        t1 = time.perf_counter()
        _, st = R.pcg(K, f, 1e-30, sample_iters)
        t2 = time.perf_counter()
        R.free_csr(K)
        R.free_mesh(m)
        return {"kind": "reference", "setup_s": t1 - t0, "solve_s": t2 - t1, "wall_s": t2 - t0,
                "iters": st["iterations"], "per_iter_s": st["t_solve"] / max(st["iterations"], 1)}
    O = oracle.Oracle()
    t0 = time.perf_counter()
    rp, cols = O.build_stiffness_pattern(mesh.num_nodes, mesh.triangles)
    kv = O.assemble_stiffness(mesh.xy, mesh.triangles, O.constitutive_matrix(1.0, 0.3), 1.0, rp, cols)
    f = np.zeros(mesh.num_dofs)
    O.add_traction(mesh.xy, mesh.triangles, mesh.boundary_edges["right"], 1.0, 1.0, 0.0, f)
    O.apply_dirichlet(rp, cols, kv, dofs, vals, f)
    t1 = time.perf_counter()
    _, st = O.pcg_jacobi(rp, cols, kv, f, 1e-30, sample_iters)
    t2 = time.perf_counter()
    return {"kind": "port", "setup_s": t1 - t0, "solve_s": t2 - t1, "wall_s": t2 - t0, "iters": st["iterations"],
            "per_iter_s": (t2 - t1) / max(st["iterations"], 1)}


def cpu_baseline_entry(s, n_dofs, rec):
    """The reference's time-to-solve on this host: its measured setup and per-iteration cost from
    the bounded sample, times the iteration count its own full run needed (the committed record)."""
    cr = rec["meta"]["cpu_run"]
    iters_full = int(rec["meta"]["iters"])
    t = s["setup_s"] + s["per_iter_s"] * iters_full
    return {"value": n_dofs / t, "unit": "DOF/s", "cores": 1, "kind": s["kind"], "time_to_solve_s": t,
            "extrapolated": True, "sample_iters": s["iters"], "iterations_full_run": iters_full,
            "sample": (f"full pattern+assembly+loads+BCs ({s['setup_s']:.2f} s) + {s['iters']} PCG iterations "
                       f"({s['per_iter_s'] * 1e3:.2f} ms each) on this host, scaled to the {iters_full} iterations "
                       f"of the reference's own full run (recursive residual < 1e-10, solver.cpp:80-82); "
                       f"single-threaded reference serial core, host has {os.cpu_count()} cores"),
            "full_run_record": {"file": rec["file"], "solve_s": cr["solve_s"], "per_iter_s": cr["per_iter_full_s"],
                                "setup_s": cr["build_stiffness_pattern_s"] + cr["assemble_stiffness_s"] +
                                cr["add_traction_s"] + cr["apply_dirichlet_s"] + cr["solver_setup_s"],
                                "host": cr["cpu_model"], "nproc": cr["nproc"], "date": cr["date"],
                                "sample_vs_full_per_iter_on_that_host": cr["sample_vs_full"]},
            "per_iter_here_vs_record_host": s["per_iter_s"] / cr["per_iter_full_s"]}


# ---- the reference arm ----------------------------------------------------------------------------

def run_reference(a, dist: Dist):
    if dist.rank != 0:
        return 0
    pkg = importlib.import_module("mpi-cst-fem-solver_b200.plate")
    n_r, n_t, desc = WORKLOADS[a.workload]
    mesh = pkg.quarter_plate(n_r, n_t)
    dofs, vals = pkg.symmetry_dirichlet(mesh)
    rec = reference_record(a.workload)
    if rec is None or "cpu_run" not in rec["meta"]:
        print(json.dumps({"impl": "reference", "unavailable": f"no full-run record of the reference for {a.workload}"}))
        return 0
    sample_iters = 50
    samples = []
    for i in range(a.warmup + a.steps):
        s = cpu_sample(mesh, dofs, vals, sample_iters)
        if i >= a.warmup:
            samples.append(s)
    per_it = statistics.median(s["per_iter_s"] for s in samples)
    setup = statistics.median(s["setup_s"] for s in samples)
    wall = statistics.median(s["wall_s"] for s in samples)
    cb = cpu_baseline_entry({"kind": samples[0]["kind"], "setup_s": setup, "per_iter_s": per_it,
                             "iters": sample_iters}, mesh.num_dofs, rec)
    cb["value_note"] = "value = this line's value"
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "DOF/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": wall * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "extrapolated": True, "sample_iters": sample_iters,
            "config": {"workload": f"{a.workload}: {desc}, {mesh.num_dofs} DOFs",
                       "step": (f"one bounded sample of the reference serial core: pattern + assembly + loads + "
                                f"BCs + {sample_iters} Jacobi-PCG iterations (ms_per_step is that sample's wall "
                                f"time); value = DOFs / (setup + per-iteration time x the "
                                f"{rec['meta']['iters']} iterations of its own full run)")},
            "cpu_baseline": cb, "time_to_solve_s": cb["time_to_solve_s"],
            "e2e": {"value": cb["value"], "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- the batched solve (64 uneven plates x 4 load cases) -------------------------------------------

def run_batch(a, pkg, sweep_shapes: bool = False, reps: int = 3):
    """64 seeded plates (n_r 20..200, n_theta = 2 n_r, a, E, nu, plane condition random) x 4 load
    cases in one persistent, graph-captured launch with the autotuned shape, against the same 256
    systems solved one at a time by the single-system mixed-precision solve."""
    import torch
    specs = pkg.plate.random_batch(count=64, seed=2026)
    t0 = time.perf_counter()
    batch = pkg.build_batch(specs)
    solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=200000))
    solver.setup(batch, device_rhs=True)
    t_setup = time.perf_counter() - t0
    shapes = {}
    if sweep_shapes:
        for c in (1, 2, 4, 8, 16):
            for t in (256, 512):
                try:
                    shapes[f"{c}x{t}"] = solver.solve(config=(c, t), device=True).seconds
                except pkg.CstgError as e:
                    shapes[f"{c}x{t}"] = str(e)
    t0 = time.perf_counter()
    cfg, t_tune = solver.autotune(max_iter=300)
    tune_s = time.perf_counter() - t0
    times = [solver.solve(device=True).seconds for _ in range(reps)]
    sol = solver.solve(device=True)
    dofs = int(batch.mesh.num_dofs)
    one, its_one = 0.0, 0
    ctx = pkg.Context(0)
    opts = pkg.SolverOptions(rtol=1e-10, max_iter=200000, precision="mixed", true_residual_stop=True)
    for s, sp in enumerate(specs):
        m = pkg.plate.quarter_plate(sp.n_r, sp.n_theta, a=sp.a)
        K = pkg.build_stiffness_pattern(m, ctx=ctx)
        pkg.assemble_stiffness(m, batch.D[s], 1.0, K)
        sl = batch.dof_range(s)
        bs = torch.from_numpy(np.ascontiguousarray(solver.b[:, sl])).to(0)
        pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, torch.zeros(m.num_dofs, dtype=torch.float64, device=0))
        cg = pkg.CgJacobiSolver(opts)
        cg.setup(K)
        x = torch.zeros(m.num_dofs, dtype=torch.float64, device=0)
        for q in range(batch.n_cases):
            st = cg.solve(bs[q].contiguous(), x)
            one += st.solve_seconds
            its_one += st.iterations
    ctx.close()
    med = statistics.median(times)
    out = {"workload": "64 plates (n_r 20..200, n_theta = 2 n_r, seed 2026) x 4 load cases (tension x, tension y, "
                       "shear, biaxial), mixed precision, rtol 1e-10 on each FP64 true residual",
           "systems": batch.n_plates * batch.n_cases, "dofs_total": dofs, "dof_cases": dofs * batch.n_cases,
           "setup_s": t_setup, "autotuned": {"cluster_ctas": cfg[0], "threads": cfg[1]}, "autotune_s": tune_s,
           "batch_solve_s": med, "batch_solve_all_s": times,
           "converged": int(np.sum(sol.converged)), "max_true_rel": float(sol.true_rel_residual.max()),
           "iterations_total": int(sol.iterations.sum()), "iterations_max": int(sol.iterations.max()),
           "one_by_one_solve_s": one, "one_by_one_iterations": its_one,
           "speedup_vs_one_by_one": one / med, "dof_cases_per_s": dofs * batch.n_cases / med}
    if shapes:
        out["shapes_s"] = shapes
    solver.close()
    return out


# ---- the large plate (the config's n_r = 800 x n_theta = 2500 O-grid) --------------------------------

def run_large(a, pkg, n_r=800, n_t=2500):
    """The learned cycle in mixed precision on the large plate against plain FP64 Jacobi-PCG on the
    same GPU (solve times, iterations, the two solutions' difference, the SCF at the hole)."""
    import torch
    m = pkg.plate.quarter_plate(n_r, n_t)
    D = pkg.constitutive_matrix(1.0, 0.3)
    ctx = pkg.Context(0)
    K = pkg.build_stiffness_pattern(m, ctx=ctx)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = torch.zeros(m.num_dofs, dtype=torch.float64, device="cuda")
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    out = {"workload": f"quarter plate O-grid n_r={n_r} x n_theta={n_t}, {m.num_dofs} DOFs, {K.nnz()} nnz"}
    xs = {}
    for name, kw in (("learned_mixed", dict(precision="mixed", preconditioner="learned_mg")),
                     ("plain_fp64", dict())):
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=400000, true_residual_stop=True, **kw))
        s.setup(K)
        if kw.get("preconditioner") == "learned_mg":
            pkg.learned.setup(K, pkg.learned.load_weights(mode="cycle"), pkg.learned.node_material(D, m.num_nodes))
            s.solve(b, torch.zeros_like(b))  # warm-up: hierarchy, graphs
        x = torch.zeros_like(b)
        st = s.solve(b, x)
        xs[name] = x
        out[name] = {"solve_s": st.solve_seconds, "iterations": st.iterations,
                     "true_rel_residual": st.true_rel_residual, "converged": st.converged}
    out["speedup_solve"] = out["plain_fp64"]["solve_s"] / out["learned_mixed"]["solve_s"]
    out["x_rel_learned_vs_plain_fp64"] = float(torch.linalg.vector_norm(xs["learned_mixed"] - xs["plain_fp64"]) /
                                               torch.linalg.vector_norm(xs["plain_fp64"]))
    strs = pkg.compute_element_stresses(ctx, xs["learned_mixed"].cpu().numpy(), 1.0, 0.3)
    out["scf"] = float(pkg.scf_at_hole(strs, 1.0)[0])
    ctx.close()
    return out


# ---- our arm --------------------------------------------------------------------------------------

def run_ours(a, dist: Dist):
    import torch
    pkg = importlib.import_module("mpi-cst-fem-solver_b200")
    dev = dist.local_rank if a.gpus > 1 else 0
    torch.cuda.set_device(dev)
    dist.init("nccl")
    L = pkg.native.load(build_if_missing=False)
    mesh, D, dofs, vals = make_inputs(pkg, a.workload)
    n_r, n_t, desc = WORKLOADS[a.workload]
    n, N = mesh.num_dofs, mesh.num_nodes
    rec = reference_record(a.workload)
    precond = PRECONDS[a.precond]
    learned_any = precond in ("learned", "learned_mg")

    stream = torch.cuda.Stream(device=dev)
    ctx = pkg.Context(dev)
    ctx.set_stream(stream)
    # device-resident inputs: mesh, the loaded edges, the prescribed DOFs
    d_xy = torch.from_numpy(mesh.xy).to(dev)
    d_tri = torch.from_numpy(mesh.triangles).to(dev)
    d_right = torch.from_numpy(np.ascontiguousarray(mesh.boundary_edges["right"].reshape(-1))).to(dev)
    d_dofs = torch.from_numpy(dofs).to(dev)
    d_vals = torch.from_numpy(vals).to(dev)
    d_b = torch.zeros(n, dtype=torch.float64, device=dev)
    d_x = torch.zeros_like(d_b)
    dmesh = pkg.plate.Mesh(xy=d_xy, triangles=d_tri, boundary_edges={"right": d_right})
    torch.cuda.synchronize()
    opts = pkg.SolverOptions(rtol=1e-10, max_iter=a.max_iter, precision=a.precision, true_residual_stop=True,
                             preconditioner=precond)
    w_cycle = pkg.learned.load_weights(mode="cycle")
    w_local = pkg.learned.load_weights(mode="local")
    weights = w_cycle if precond == "learned_mg" else w_local
    mat = pkg.learned.node_material(D, N)
    last = {}

    def system():  # pattern, assembly, loads and Dirichlet on the GPU (on the caller's stream)
        K = pkg.build_stiffness_pattern(dmesh, ctx=ctx)
        pkg.assemble_stiffness(dmesh, D, 1.0, K)
        d_b.zero_()
        pkg.add_traction(K, d_right, 1.0, 1.0, 0.0, d_b)  # loads on the GPU (bc.cpp:190-253)
        pkg.apply_dirichlet((d_dofs, d_vals), K, d_b)
        return K

    def step():
        with torch.cuda.stream(stream):
            K = system()
            s = pkg.CgJacobiSolver(opts)
            s.setup(K)
            if learned_any:
                pkg.learned.setup(K, weights, mat)
            last["st"] = s.solve(d_b, d_x)
            last["K"] = K

    def ev_start():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    def ev_stop(e0):
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    sync = torch.cuda.synchronize
    if a.only:
        out = run_only(a, pkg, step, system, last, ctx, stream, ev_start, ev_stop, d_b, D, N, n, w_cycle)
        print(json.dumps(out))
        ctx.close()
        return 0

    clocks = ClockSampler(dev)
    for _ in range(a.warmup):
        step()
    sync()
    l0 = L.cstg_kernel_launches()
    clocks.start()
    el = timed_region(step, a.steps, 0, dist, ev_start, ev_stop, sync)
    clk = clocks.stop()
    launches = L.cstg_kernel_launches() - l0
    el_max = dist.max(el, device=f"cuda:{dev}")
    st = last["st"]
    if not st.converged or not st.true_rel_residual < 1e-10:
        raise RuntimeError(f"solve did not reach the FP64 true residual 1e-10: {st.message}, "
                           f"true {st.true_rel_residual:.3e}")
    t_step = el_max / a.steps
    value = a.gpus * n / t_step
    K = last["K"]
    x_head = d_x.cpu().numpy()
    line = {
        "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f32 (SpMV, cycle operators) + f64 (vectors, scalars, reliable updates) + bf16 (network)"
                  if learned_any and a.precision == "mixed" else
                  "f32 (SpMV) + f64" if a.precision == "mixed" else "f64"),
        "data": "synthetic",
        "config": {"workload": f"{a.workload}: {desc}, {n} DOFs, {K.nnz()} nnz, E=1 nu=0.3 plane stress t=1, "
                               "traction (1,0) on x=10, u_x=0 on x=0, u_y=0 on y=0",
                   "step": (f"pattern + assembly + traction loads (GPU) + Dirichlet + Jacobi setup + {a.precond} "
                            "preconditioner setup + flexible CG to rtol 1e-10 on the FP64 true residual"),
                   "preconditioner": a.precond, "precision": a.precision, "dofs": n, "nnz": K.nnz(),
                   "l2": f"inputs larger than L2 (FP64 matrix values {K.nnz() * 8 / 1e6:.0f} MB)",
                   "parallelism": f"replicas x{a.gpus}"},
        "time_to_solve_s": t_step, "iterations": st.iterations, "refinements": st.refinements,
        "true_rel_residual": st.true_rel_residual, "solve_s": st.solve_seconds, "message": st.message,
        "x_rel_vs_reference_u": rel_error_vs_reference(rec, x_head),
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if rec is not None:
        line["reference_run"] = {"iterations": rec["meta"]["iters"], "true_rel_residual": rec["meta"]["true_rel"],
                                 "scf": rec["meta"]["scf"], "file": rec["file"],
                                 "u_compared": "every 8th node" if rec["idx"] is not None else "all DOFs"}
    strs = pkg.compute_element_stresses(ctx, x_head, 1.0, 0.3)
    scf, scf_elem = pkg.scf_at_hole(strs, 1.0)
    line["scf"] = {"value": scf, "element": scf_elem, "analytic_infinite_plate": 3.0,
                   "reference": rec["meta"]["scf"] if rec else None}

    if not a.no_compare:
        line.update(compare_solves(a, pkg, K, d_b, d_x, stream, rec, st, t_step, mat, w_cycle))
    line.update(rooflines(a, pkg, K, ctx, stream, ev_start, ev_stop, N, n, mat, weights, precond))
    if not a.no_e2e:
        line["e2e"] = run_e2e(a, pkg, dist, dev, mesh, D, dofs, vals, opts, weights, mat, learned_any, sync)
    if dist.rank == 0 and not a.no_cpu_baseline and a.gpus == 1 and rec is not None and "cpu_run" in rec["meta"]:
        s = cpu_sample(mesh, dofs, vals, a.cpu_sample_iters)
        line["cpu_baseline"] = cpu_baseline_entry(s, n, rec)
    if dist.rank == 0 and not a.no_batch and a.gpus == 1:
        line["batch"] = run_batch(a, pkg)
    if dist.rank == 0 and not a.no_large and a.gpus == 1:
        line["large_plate"] = run_large(a, pkg)
    ctx.close()
    if dist.rank == 0:
        print(json.dumps(line))
    dist.close()
    return 0


def compare_solves(a, pkg, K, d_b, d_x, stream, rec, st_head, t_step, mat, w_cycle):
    """The comparison solves on the step's matrix (not in `value`), each with its error against the
    reference's displacements:
      reference_rule  FP64 Jacobi-PCG under the reference's own stopping rule (recursive residual,
                      solver.cpp:80-82): iterations against the reference's full run
      plain_fp64      FP64 Jacobi-PCG to the FP64 true residual: the plain GPU Jacobi-PCG
      jacobi_mixed    Jacobi-PCG with FP32 SpMV, FP64 vectors/scalars and reliable updates
      amg_mixed       the Chebyshev multigrid cycle (no network), flexible CG, mixed
      learned_zero    the learned cycle with the network at zero (its post-smoother is one damped
                      Jacobi step): the method without the trained network"""
    import torch
    out = {}

    def solve_with(name, setup=None, **kw):
        x = torch.zeros_like(d_x)
        with torch.cuda.stream(stream):
            s_ = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=400000, **kw))
            s_.setup(K)
            if setup:
                setup()
            if kw.get("preconditioner", "jacobi") != "jacobi":
                s_.solve(d_b, x)  # warm-up: hierarchy, graph capture
            t0 = time.perf_counter()
            st = s_.solve(d_b, x)
            wall = time.perf_counter() - t0
        torch.cuda.synchronize()
        xh = x.cpu().numpy()
        out[name] = {"solve_s": st.solve_seconds, "wall_s": wall, "iterations": st.iterations,
                     "refinements": st.refinements, "true_rel_residual": st.true_rel_residual,
                     "converged": st.converged, "x_rel_vs_reference_u": rel_error_vs_reference(rec, xh)}
        return st

    st_ref = solve_with("reference_rule")
    if rec is not None:
        out["reference_rule"]["iterations_reference_run"] = rec["meta"]["iters"]
    st_64 = solve_with("plain_fp64", true_residual_stop=True)
    solve_with("jacobi_mixed", precision="mixed", true_residual_stop=True)
    solve_with("amg_mixed", precision="mixed", preconditioner="amg", true_residual_stop=True)
    zero = np.zeros_like(w_cycle)
    st_z = solve_with("learned_zero", setup=lambda: pkg.learned.setup(K, zero, mat), precision="mixed",
                      preconditioner="learned_mg", true_residual_stop=True)
    st_64s = st_64.solve_seconds
    out["speedup"] = {
        "headline_step_vs_plain_fp64_solve": st_64s / t_step,
        "headline_solve_vs_plain_fp64_solve": st_64s / st_head.solve_seconds,
        "iterations_plain_fp64": st_64.iterations, "iterations_headline": st_head.iterations,
        "iteration_ratio": st_64.iterations / max(st_head.iterations, 1),
        "time_per_iteration_ratio": (st_head.solve_seconds / max(st_head.iterations, 1)) /
                                    (st_64s / max(st_64.iterations, 1)),
        "network_vs_zero_network_iterations": (st_head.iterations, st_z.iterations),
        "note": "speedup = iteration_ratio / time_per_iteration_ratio (solve); the step adds pattern, assembly, "
                "loads, Dirichlet and every setup"}
    return out


def rooflines(a, pkg, K, ctx, stream, ev_start, ev_stop, N, n, mat, weights, precond):
    """The dominant kernel of the step (the network's message-passing layer for the learned
    preconditioners) and the two SpMVs, timed alone with CUDA events on the context's stream."""
    import torch
    peak, peak_kind = measured_peaks()
    peak_note = f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    full = a.workload == "plate2m"
    nnz = K.nnz()
    nb = nnz // 4
    noff = nb - N

    def roof(kernel, nbytes, seconds, traffic=None, **extra):
        return {"bound": "hbm", "kernel": kernel, "achieved": nbytes / seconds / 1e9, "peak": peak, "unit": "GB/s",
                "frac": nbytes / seconds / 1e9 / peak, "peak_kind": peak_note, "traffic": traffic,
                "algorithmic_bytes": nbytes, "launch_us": seconds * 1e6, **extra}

    def time_launches(fn, reps=100):
        with torch.cuda.stream(stream):
            for _ in range(10):
                fn()
            e0 = ev_start()
            for _ in range(reps):
                fn()
            return ev_stop(e0) / reps

    xs = torch.randn(n, dtype=torch.float64, device=K.ctx.device)
    ys = torch.empty_like(xs)
    with torch.cuda.stream(stream):
        s0 = pkg.CgJacobiSolver()
        s0.setup(K)
    spmv64_bytes = nnz * 8 + nb * 4 + (N + 1) * 4 + n * 8 + n * 8
    spmv32_bytes = noff * (16 + 4) + N * 32 + (N + 1) * 4 + n * 8 + n * 8
    r64 = roof("k_spmv_block (FP64 2x2-block SpMV)", spmv64_bytes, time_launches(lambda: K.multiply(xs, ys)),
               profile_traffic("spmv_block_fp64_plate2m.md") if full else None)
    r32 = roof("k_spmv_mixed (FP32 difference-form 2x2-block SpMV, FP64 vectors)", spmv32_bytes,
               time_launches(lambda: K.multiply_mixed(xs, ys)),
               profile_traffic("spmv_mixed_f32_plate2m.md") if full else None)
    out = {"spmv_fp64": r64, "spmv_mixed": r32}
    # the network's layer: H in (128 B / node, BF16) once, H out, and the graph once: with a gather
    # plan (every tile of the O-grid plates) the node slots (16 B / node) and the tiles' runs
    # (80 B / tile), else the node pointers and neighbour indices
    with torch.cuda.stream(stream):
        pkg.learned.setup(K, weights, mat)
        tm = pkg.learned.time_stages(K, reps=50)
    planned = os.environ.get("CSTG_MP_GATHER", "") != "rows"
    tiles = (N + 127) // 128
    graph_bytes = N * 16 + tiles * 80 if planned else (N + 1) * 4 + nb * 4
    layer_bytes = N * 2 * 128 + graph_bytes
    last_bytes = N * 128 + graph_bytes + n * 8 * 3  # H in; r, D^-1 in, z out
    enc_bytes = N * (16 + 24 + 128)
    lay = roof(("k_mp_layer_ws (message-passing layer, warp-specialised, tcgen05 BF16, layer 2 of 3, gather plan)"
                if planned else "k_mp_layer_tc (message-passing layer, tcgen05 BF16, layer 2 of 3, row gather)"),
               layer_bytes, tm["layer_s"][1],
               profile_traffic("mp_layer_ws_plate2m.md") if full and planned else None,
               layers_us=[t * 1e6 for t in tm["layer_s"]], encoder_us=tm["encoder_s"] * 1e6,
               last_layer_gbs=last_bytes / tm["layer_s"][2] / 1e9, encoder_gbs=enc_bytes / tm["encoder_s"] / 1e9,
               network_apply_us=(tm["encoder_s"] + sum(tm["layer_s"])) * 1e6)
    out["network"] = lay
    if precond in ("learned", "learned_mg"):
        out["roofline"] = lay
    elif precond == "amg":
        with torch.cuda.stream(stream):
            tma = pkg.amg_time(K, reps=50)
        out["roofline"] = roof("k_amg_sweep_f32 (finest-level smoothing step)", spmv32_bytes + 2 * n * 8,
                               tma["sweep_s"], profile_traffic("amg_sweep_f32_plate2m.md") if full else None)
    else:
        out["roofline"] = r32 if a.precision == "mixed" else r64
    return out


def run_e2e(a, pkg, dist, dev, mesh, D, dofs, vals, opts, weights, mat, learned_any, sync):
    """The step through the C ABI with pinned host buffers: mesh, loaded edges and BCs up, the
    traction loads and the elimination through the host-pointer calls, displacements down."""
    import torch

    def pinned(arr):
        t = torch.empty(arr.shape, dtype={np.float64: torch.float64, np.int32: torch.int32,
                                          np.float32: torch.float32}[arr.dtype.type], pin_memory=True)
        v = t.numpy()
        v[...] = arr
        return v
    hmesh = pkg.plate.Mesh(xy=pinned(mesh.xy), triangles=pinned(mesh.triangles),
                           boundary_edges={"right": pinned(np.ascontiguousarray(mesh.boundary_edges["right"]))})
    h_dofs, h_vals = pinned(dofs), pinned(vals)
    h_b = pinned(np.zeros(mesh.num_dofs))
    h_x = pinned(np.zeros(mesh.num_dofs))
    h_mat = pinned(np.ascontiguousarray(mat))
    ectx = pkg.Context(dev)
    last = {}

    def e2e_step():
        K2 = pkg.build_stiffness_pattern(hmesh, ctx=ectx)
        pkg.assemble_stiffness(hmesh, D, 1.0, K2)
        h_b.fill(0.0)
        pkg.add_traction(K2, hmesh.boundary_edges["right"], 1.0, 1.0, 0.0, h_b)
        pkg.apply_dirichlet((h_dofs, h_vals), K2, h_b)
        s2 = pkg.CgJacobiSolver(opts)
        s2.setup(K2)
        if learned_any:
            pkg.learned.setup(K2, weights, h_mat)
        last["st"] = s2.solve(h_b, h_x)

    def wall_start():
        return time.perf_counter()

    def wall_stop(t0):
        return time.perf_counter() - t0

    el2 = timed_region(e2e_step, a.steps, a.warmup, dist, wall_start, wall_stop, sync)
    el2 = dist.max(el2, device=f"cuda:{dev}")
    h2d = mesh.xy.nbytes + mesh.triangles.nbytes + mesh.boundary_edges["right"].nbytes + dofs.nbytes + vals.nbytes \
        + h_b.nbytes + mat.nbytes
    d2h = h_b.nbytes + h_x.nbytes
    ectx.close()
    return {"value": a.gpus * mesh.num_dofs / (el2 / a.steps), "unit": "DOF/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": el2 / a.steps * 1e3,
            "converged": bool(last["st"].converged),
            "path": "C ABI, host pinned buffers (cstg_set_mesh .. cstg_pcg_solve)"}


def run_only(a, pkg, step, system, last, ctx, stream, ev_start, ev_stop, d_b, D, N, n, w_cycle):
    import torch
    out = {"mode": a.only, "workload": a.workload}
    if a.only == "batch":
        out.update(run_batch(a, pkg, sweep_shapes=True, reps=a.reps))
        return out
    if a.only == "network":  # the assembled system and the network's stages alone, no solve before
        with torch.cuda.stream(stream):
            K = system()
            pkg.CgJacobiSolver().setup(K)
            pkg.learned.setup(K, w_cycle, pkg.learned.node_material(D, N))
            out.update(pkg.learned.time_stages(K, reps=a.reps))
        return out
    step()
    torch.cuda.synchronize()
    K = last["K"]
    if a.only == "solve":
        out.update(iterations=last["st"].iterations, solve_s=last["st"].solve_seconds, message=last["st"].message)
    elif a.only == "learned":
        with torch.cuda.stream(stream):
            pkg.learned.setup(K, w_cycle, pkg.learned.node_material(D, N))
            out.update(pkg.learned.time_stages(K, reps=a.reps))
    elif a.only == "amg":
        with torch.cuda.stream(stream):
            info = pkg.amg_setup(K)
            tm = pkg.amg_time(K, reps=max(a.reps, 3))
        out.update(levels=info["levels"], dofs=info["dofs"], setup_s=info["setup_seconds"],
                   fine_sweep_us=tm["sweep_s"] * 1e6, vcycle_us=tm["vcycle_s"] * 1e6)
    else:  # `reps` SpMV launches of the precision asked for on the assembled, eliminated matrix
        with torch.cuda.stream(stream):
            xs = torch.randn(n, dtype=torch.float64, device=K.ctx.device)
            ys = torch.empty_like(xs)
            mul = K.multiply_mixed if a.precision == "mixed" else K.multiply
            mul(xs, ys)
            e0 = ev_start()
            for _ in range(a.reps):
                mul(xs, ys)
            out["spmv_us"] = ev_stop(e0) / a.reps * 1e6
    return out


def main():
    a = parse()
    dist = Dist()
    if a.impl == "reference":
        return run_reference(a, dist)
    return run_ours(a, dist)


if __name__ == "__main__":
    sys.exit(main())
