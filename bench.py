#!/usr/bin/env python
"""Time-to-solve benchmark of the CST assembly -> Dirichlet -> Jacobi-PCG path on B200.

A step is one full pass of the path over one synthetic plate: stiffness pattern, assembly,
Dirichlet elimination, Jacobi setup and PCG to rtol 1e-10 on the FP64 TRUE residual
(||b - A x|| / ||b||). The default workload is the 2M-DOF quarter plate (O-grid n_r = 565 x
n_theta = 1766, 2,000,244 DOFs, ~28M nonzeros; E = 1, nu = 0.3, plane stress, t = 1,
traction (1, 0) on x = 10, u_x = 0 on x = 0, u_y = 0 on y = 0).

  value  DOFs solved per second with the mesh, loads and BCs already in HBM (CUDA events on
         the work stream), summed over all GPUs (independent replicas, weak scaling).
  e2e    the same through the C ABI with pinned HOST buffers: every step uploads the mesh,
         loads and BCs and downloads the displacements (wall clock around the step).

One JSON line on rank 0. `--impl reference` times the reference's own CPU path (compiled from
its sources into oracle/_ref) on this host's cores instead, on bounded samples.
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

# FP64 Jacobi-PCG iterations to the reference's own stopping rule (recursive residual < 1e-10,
# solver.cpp:80-82) on each workload, measured with this library's FP64 solver (same
# recurrence; the GPU-vs-reference parity tests hold the count to 2 %). The CPU baseline and
# the reference arm time a bounded number of the reference's iterations and scale to this.
REF_RULE_ITERS = {"plate2m": 19530, "plate1m": 13812, "plate4m": 27665, "plate40x80": 897}

METRIC = ("time-to-solve @rtol 1e-10 (FP64 true residual), 2M-DOF plate, as DOFs solved per "
          "second")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plate2m", choices=sorted(WORKLOADS))
    ap.add_argument("--precond", default="amg", choices=["amg", "jacobi", "learned"],
                    help="preconditioner of the timed solve: smoothed-aggregation multigrid (default), "
                         "Jacobi (the reference's method, persistent kernel) or the learned network")
    ap.add_argument("--amg-smoother", default="chebyshev", choices=["chebyshev", "jacobi"],
                    help="smoother of the multigrid cycle")
    ap.add_argument("--amg-theta", type=float, nargs=2, default=[0.0, 0.03], metavar=("FINE", "COARSE"),
                    help="strength-of-connection thresholds of the multigrid aggregation")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="outer CG precision; default fp64 with amg (its finest smoother is FP32 already), "
                         "mixed otherwise")
    ap.add_argument("--cpu-sample-iters", type=int, default=150)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner comparison")
    ap.add_argument("--only", choices=["spmv", "solve", "batch", "batchsolve", "learned", "amg"], default=None,
                    help="profiling modes: `spmv` runs --reps SpMV launches on the assembled plate, "
                         "`solve` one full step, `batch` the 64-plate x 4-load-case batched solve "
                         "(every launch shape, autotuned, --reps graph replays, and the same systems "
                         "solved one by one), `batchsolve` one batched solve (8 x 512 shape) of "
                         "--batch-plates plates with n_r up to --batch-nr-max, `learned` --reps "
                         "applications of the learned preconditioner on the plate; each prints one "
                         "JSON line")
    ap.add_argument("--batch-plates", type=int, default=64)
    ap.add_argument("--batch-nr-max", type=int, default=200)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--max-iter", type=int, default=200000,
                    help="iteration cap of the solves (profiling captures use a small cap)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    if a.precision is None:
        a.precision = "fp64" if a.precond == "amg" else "mixed"
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
                 "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
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
        _, st = R.pcg(K, f, 1e-10, sample_iters)
        t2 = time.perf_counter()
        R.free_csr(K)
        R.free_mesh(m)
        return {"kind": "reference", "setup_s": t1 - t0, "solve_s": t2 - t1,
                "iters": st["iterations"], "per_iter_s": st["t_solve"] / max(st["iterations"], 1)}
    O = oracle.Oracle()
    t0 = time.perf_counter()
    rp, cols = O.build_stiffness_pattern(mesh.num_nodes, mesh.triangles)
    kv = O.assemble_stiffness(mesh.xy, mesh.triangles, O.constitutive_matrix(1.0, 0.3), 1.0, rp, cols)
    f = np.zeros(mesh.num_dofs)
    O.add_traction(mesh.xy, mesh.triangles, mesh.boundary_edges["right"], 1.0, 1.0, 0.0, f)
    O.apply_dirichlet(rp, cols, kv, dofs, vals, f)
    t1 = time.perf_counter()
    _, st = O.pcg_jacobi(rp, cols, kv, f, 1e-10, sample_iters)
    t2 = time.perf_counter()
    return {"kind": "port", "setup_s": t1 - t0, "solve_s": t2 - t1, "iters": st["iterations"],
            "per_iter_s": (t2 - t1) / max(st["iterations"], 1)}


def cpu_baseline_entry(s, n_dofs, iters_full, sample_iters):
    t = s["setup_s"] + s["per_iter_s"] * iters_full
    return {"value": n_dofs / t, "unit": "DOF/s", "cores": 1, "kind": s["kind"],
            "time_to_solve_s": t,
            "sample": (f"full pattern+assembly+loads+BCs ({s['setup_s']:.2f} s) + {s['iters']} of "
                       f"{iters_full} PCG iterations ({s['per_iter_s'] * 1e3:.2f} ms each, the "
                       f"reference's recursive-residual rule), extrapolated; single-threaded "
                       f"reference serial core, host has {os.cpu_count()} cores")}


# ---- the reference arm ----------------------------------------------------------------------------

def run_reference(a, dist: Dist):
    if dist.rank != 0:
        return 0
    pkg = importlib.import_module("mpi-cst-fem-solver_b200.plate")
    n_r, n_t, desc = WORKLOADS[a.workload]
    mesh = pkg.quarter_plate(n_r, n_t)
    dofs, vals = pkg.symmetry_dirichlet(mesh)
    iters_full = REF_RULE_ITERS.get(a.workload)
    if iters_full is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no iteration count recorded for {a.workload}"}))
        return 0
    sample_iters = max(10, a.cpu_sample_iters // 3)
    samples = []
    for i in range(a.warmup + a.steps):
        s = cpu_sample(mesh, dofs, vals, sample_iters)
        if i >= a.warmup:
            samples.append(s)
    per_it = statistics.median(s["per_iter_s"] for s in samples)
    setup = statistics.median(s["setup_s"] for s in samples)
    t = setup + per_it * iters_full
    value = mesh.num_dofs / t
    cb = cpu_baseline_entry({"kind": samples[0]["kind"], "setup_s": setup, "per_iter_s": per_it,
                             "iters": sample_iters}, mesh.num_dofs, iters_full, sample_iters)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{a.workload}: {desc}, {mesh.num_dofs} DOFs",
                       "step": "reference serial core: pattern + assembly + loads + BCs + Jacobi-PCG "
                               "(rtol 1e-10, its recursive-residual rule), bounded sample extrapolated"},
            "cpu_baseline": cb, "time_to_solve_s": t,
            "e2e": {"value": value, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- our arm --------------------------------------------------------------------------------------

def run_batch(a, pkg):
    """64 seeded plates (n_r 20..200, n_theta = 2 n_r) x 4 load cases: one batched persistent
    launch (autotuned shape) against the same 256 systems solved one at a time."""
    import torch
    specs = pkg.plate.random_batch(count=64, seed=2026)
    t0 = time.perf_counter()
    batch = pkg.build_batch(specs)
    solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=200000))
    solver.setup(batch, device_rhs=True)
    t_setup = time.perf_counter() - t0
    print(f"batch setup {t_setup:.2f} s, {batch.mesh.num_dofs} DOFs", file=sys.stderr, flush=True)
    shapes = {}
    for c in (1, 2, 4, 8, 16):
        for t in (256, 512):
            try:
                shapes[f"{c}x{t}"] = solver.solve(config=(c, t), device=True).seconds
            except pkg.CstgError as e:
                shapes[f"{c}x{t}"] = str(e)
            print(f"shape {c}x{t}: {shapes[f'{c}x{t}']}", file=sys.stderr, flush=True)
    t0 = time.perf_counter()
    cfg, t_tune = solver.autotune(max_iter=300)
    print(f"autotune {cfg} in {time.perf_counter() - t0:.2f} s", file=sys.stderr, flush=True)
    times = [solver.solve(device=True).seconds for _ in range(a.reps)]
    sol = solver.solve(device=True)
    dofs = int(batch.mesh.num_dofs)
    # the same systems one at a time through the single-system persistent solve
    one, its_one = 0.0, 0
    ctx = pkg.Context(0)
    opts = pkg.SolverOptions(rtol=1e-10, max_iter=200000, precision="mixed", true_residual_stop=True)
    for s, sp in enumerate(specs):
        m = pkg.plate.quarter_plate(sp.n_r, sp.n_theta, a=sp.a)
        K = pkg.build_stiffness_pattern(m, ctx=ctx)
        pkg.assemble_stiffness(m, batch.D[s], 1.0, K)
        sl = batch.dof_range(s)
        bs = torch.from_numpy(np.ascontiguousarray(solver.b[:, sl])).to(0)
        pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K,
                            torch.zeros(m.num_dofs, dtype=torch.float64, device=0))
        cg = pkg.CgJacobiSolver(opts)
        cg.setup(K)
        x = torch.zeros(m.num_dofs, dtype=torch.float64, device=0)
        for q in range(batch.n_cases):
            st = cg.solve(bs[q].contiguous(), x)
            one += st.solve_seconds
            its_one += st.iterations
    ctx.close()
    out = {"mode": "batch", "workload": "64 plates (n_r 20..200, seed 2026) x 4 load cases",
           "systems": batch.n_plates * batch.n_cases, "dofs_total": dofs, "dof_cases": dofs * batch.n_cases,
           "setup_s": t_setup, "shapes_s": shapes, "autotuned": list(cfg), "tune_best_s": t_tune,
           "batch_solve_s": statistics.median(times), "batch_solve_all_s": times,
           "converged": int(np.sum(sol.converged)), "max_true_rel": float(sol.true_rel_residual.max()),
           "iterations_total": int(sol.iterations.sum()), "iterations_max": int(sol.iterations.max()),
           "fp64_switched_plates": int(np.sum(sol.fp64[:, 0])),
           "refinements_total": int(sol.refinements.sum()),
           "one_by_one_solve_s": one, "one_by_one_iterations": its_one,
           "dof_cases_per_s": dofs * batch.n_cases / statistics.median(times)}
    solver.close()
    return out


def run_ours(a, dist: Dist):
    import torch
    pkg = importlib.import_module("mpi-cst-fem-solver_b200")
    dev = dist.local_rank if a.gpus > 1 else 0
    torch.cuda.set_device(dev)
    dist.init("nccl")
    L = pkg.native.load(build_if_missing=False)
    mesh, D, dofs, vals = make_inputs(pkg, a.workload)
    n_r, n_t, desc = WORKLOADS[a.workload]
    n = mesh.num_dofs

    stream = torch.cuda.Stream(device=dev)
    ctx = pkg.Context(dev)
    ctx.set_stream(stream)
    smoother_code = {"chebyshev": pkg.native.AMG_CHEBYSHEV, "jacobi": pkg.native.AMG_JACOBI}[a.amg_smoother]
    ctx.check(ctx.L.cstg_amg_set_smoother(ctx.h, smoother_code))
    ctx.check(ctx.L.cstg_amg_set_strength(ctx.h, *a.amg_theta))
    # loads on the host (bc.cpp:190-253) once; the step starts from them
    ctx.set_mesh(mesh)
    b0 = np.zeros(n)
    pkg.add_traction(ctx, mesh.boundary_edges["right"], 1.0, 1.0, 0.0, b0)

    # device-resident inputs
    d_xy = torch.from_numpy(mesh.xy).to(dev)
    d_tri = torch.from_numpy(mesh.triangles).to(dev)
    d_dofs = torch.from_numpy(dofs).to(dev)
    d_vals = torch.from_numpy(vals).to(dev)
    d_b0 = torch.from_numpy(b0).to(dev)
    d_b = torch.empty_like(d_b0)
    d_x = torch.empty_like(d_b0)
    dmesh = pkg.plate.Mesh(xy=d_xy, triangles=d_tri, boundary_edges=mesh.boundary_edges)
    torch.cuda.synchronize()
    opts = pkg.SolverOptions(rtol=1e-10, max_iter=a.max_iter, precision=a.precision, true_residual_stop=True,
                             preconditioner=a.precond)
    last = {}
    l_weights = pkg.learned.load_weights()
    l_mat = pkg.learned.node_material(D, mesh.num_nodes)

    def step():
        with torch.cuda.stream(stream):
            K = pkg.build_stiffness_pattern(dmesh, ctx=ctx)
            pkg.assemble_stiffness(dmesh, D, 1.0, K)
            d_b.copy_(d_b0)
            pkg.apply_dirichlet((d_dofs, d_vals), K, d_b)
            s = pkg.CgJacobiSolver(opts)
            s.setup(K)
            if a.precond == "learned":
                pkg.learned.setup(K, l_weights, l_mat)
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
        out = {"mode": a.only, "workload": a.workload}
        if a.only == "batch":
            out = run_batch(a, pkg)
        elif a.only == "batchsolve":
            specs = pkg.plate.random_batch(count=a.batch_plates, seed=2026, n_r_range=(20, a.batch_nr_max))
            solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=200000))
            solver.setup(pkg.build_batch(specs), device_rhs=True)
            sol = solver.solve(config=(8, 512), device=True)
            out.update(plates=a.batch_plates, seconds=sol.seconds, converged=int(sol.converged.sum()),
                       iterations_max=int(sol.iterations.max()))
            solver.close()
        elif a.only == "amg":
            with torch.cuda.stream(stream):
                K = pkg.build_stiffness_pattern(dmesh, ctx=ctx)
                pkg.assemble_stiffness(dmesh, D, 1.0, K)
                d_b.copy_(d_b0)
                pkg.apply_dirichlet((d_dofs, d_vals), K, d_b)
                pkg.CgJacobiSolver().setup(K)
                info = pkg.amg_setup(K)
                z = torch.empty_like(d_b)
                pkg.amg_apply(K, d_b, z)
                e0 = ev_start()
                for _ in range(a.reps):
                    pkg.amg_apply(K, d_b, z)
                out.update(vcycle_us=ev_stop(e0) / a.reps * 1e6, levels=info["levels"], dofs=info["dofs"],
                           nnz=info["nnz"], setup_s=info["setup_seconds"])
                tm = pkg.amg_time(K, reps=max(a.reps, 3))
                pkg.amg_set_tail(K, False)
                tm2 = pkg.amg_time(K, reps=max(a.reps, 3))
                pkg.amg_set_tail(K, True)
                info2 = pkg.amg_setup(K)  # a rebuild on the same context (buffers reused)
                out.update(fine_sweep_us=tm["sweep_s"] * 1e6, vcycle_timed_us=tm["vcycle_s"] * 1e6,
                           vcycle_level_by_level_us=tm2["vcycle_s"] * 1e6, tail_level=info["tail_level"],
                           tail_cluster=info["tail_cluster"], rebuild_s=info2["setup_seconds"])
        elif a.only == "learned":
            with torch.cuda.stream(stream):
                K = pkg.build_stiffness_pattern(dmesh, ctx=ctx)
                pkg.assemble_stiffness(dmesh, D, 1.0, K)
                d_b.copy_(d_b0)
                pkg.apply_dirichlet((d_dofs, d_vals), K, d_b)
                pkg.CgJacobiSolver().setup(K)
                pkg.learned.setup(K, pkg.learned.load_weights(), pkg.learned.node_material(D, mesh.num_nodes))
                z = torch.empty_like(d_b)
                pkg.learned.apply(K, d_b, z)
                e0 = ev_start()
                for _ in range(a.reps):
                    pkg.learned.apply(K, d_b, z)
                out["apply_us"] = ev_stop(e0) / a.reps * 1e6
        elif a.only == "solve":
            step()
            sync()
            out.update(iterations=last["st"].iterations, solve_s=last["st"].solve_seconds)
        else:  # the assembled, eliminated matrix and `reps` plain SpMV launches, nothing else
            with torch.cuda.stream(stream):
                K = pkg.build_stiffness_pattern(dmesh, ctx=ctx)
                pkg.assemble_stiffness(dmesh, D, 1.0, K)
                d_b.copy_(d_b0)
                pkg.apply_dirichlet((d_dofs, d_vals), K, d_b)
                xs = torch.randn(n, dtype=torch.float64, device=dev)
                ys = torch.empty_like(xs)
                e0 = ev_start()
                if a.precision == "mixed":
                    pkg.CgJacobiSolver().setup(K)
                    K.multiply_mixed(xs, ys)  # builds the FP32 operator (untimed)
                    e0 = ev_start()
                    for _ in range(a.reps):
                        K.multiply_mixed(xs, ys)
                else:
                    for _ in range(a.reps):
                        K.multiply(xs, ys)
                out["spmv_us"] = ev_stop(e0) / a.reps * 1e6
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

    # comparison solves on the same matrix (not in `value`):
    #   ref_rule      FP64 Jacobi-PCG under the reference's own stopping rule (recursive residual,
    #                 solver.cpp:80-82): its iteration count scales the CPU baseline
    #   plain_fp64    FP64 Jacobi-PCG to the FP64 true residual: the plain GPU Jacobi-PCG
    #   jacobi_mixed  Jacobi-PCG with the FP32 SpMV and preconditioner, FP64 scalars and
    #                 true-residual refinement (the persistent kernel)
    #   learned_mixed the learned preconditioner (packaged weights) in flexible CG, mixed SpMV
    K = last["K"]

    def solve_with(x_out=None, **kw):
        s_ = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=400000, **kw))
        s_.setup(K)
        return s_, s_.solve(d_b, torch.empty_like(d_x) if x_out is None else x_out)

    x_ref = torch.empty_like(d_x)
    with torch.cuda.stream(stream):
        s_ref, st_ref = solve_with(x_ref)
        _, st_64 = solve_with(true_residual_stop=True)
        _, st_jm = solve_with(precision="mixed", true_residual_stop=True)
    sync()

    learned = None
    if not a.no_learned:
        with torch.cuda.stream(stream):
            s_l = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=200000, precision="mixed",
                                                       preconditioner="learned", true_residual_stop=True))
            s_l.setup(K)
            t0 = time.perf_counter()
            pkg.learned.setup(K, l_weights, l_mat)
            t_setup = time.perf_counter() - t0
            s_l.solve(d_b, torch.empty_like(d_x))  # warm-up (graph capture)
            st_l = s_l.solve(d_b, torch.empty_like(d_x))
        sync()
        learned = {"solve_s": st_l.solve_seconds, "setup_s": t_setup, "iterations": st_l.iterations,
                   "true_rel_residual": st_l.true_rel_residual, "converged": st_l.converged,
                   "speedup_vs_plain_fp64": st_64.solve_seconds / st_l.solve_seconds,
                   "message": st_l.message}

    # dominant kernels timed alone (CUDA events, back-to-back launches)
    N = mesh.num_nodes
    nnz = K.nnz()
    nb = nnz // 4
    noff = nb - N
    reps = 100

    def time_launches(fn):
        with torch.cuda.stream(stream):
            for _ in range(20):
                fn()
            e0 = ev_start()
            for _ in range(reps):
                fn()
            return ev_stop(e0) / reps

    peak, peak_kind = measured_peaks()
    peak_note = f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    full = a.workload == "plate2m"

    def roof(kernel, nbytes, seconds, traffic=None, **extra):
        return {"bound": "hbm", "kernel": kernel, "achieved": nbytes / seconds / 1e9, "peak": peak, "unit": "GB/s",
                "frac": nbytes / seconds / 1e9 / peak, "peak_kind": peak_note, "traffic": traffic,
                "algorithmic_bytes": nbytes, "launch_us": seconds * 1e6, **extra}

    xs = torch.randn(n, dtype=torch.float64, device=dev)
    ys = torch.empty_like(xs)
    spmv64_s = time_launches(lambda: K.multiply(xs, ys))
    spmv64_bytes = nnz * 8 + nb * 4 + (N + 1) * 4 + n * 8 + n * 8
    roof64 = roof("k_spmv_block (FP64 2x2-block SpMV)", spmv64_bytes, spmv64_s,
                  profile_traffic("spmv_block_fp64_plate2m.md") if full else None)
    with torch.cuda.stream(stream):
        s_ref.setup(K)  # the FP32 operator of this matrix
    spmv32_s = time_launches(lambda: K.multiply_mixed(xs, ys))
    spmv32_bytes = noff * (16 + 4) + N * 32 + (N + 1) * 4 + n * 8 + n * 8
    roof32 = roof("k_spmv_mixed (FP32 difference-form 2x2-block SpMV, FP64 vectors)", spmv32_bytes, spmv32_s,
                  profile_traffic("spmv_mixed_f32_plate2m.md") if full else None)

    # The persistent Jacobi-PCG kernel (one cooperative launch runs every iteration): algorithmic
    # bytes per launch = the 3-pass iteration model (SpMV + x/r update + p update) x iterations.
    def persistent_roof(stx, precision):
        it_bytes = (spmv32_bytes if precision == "mixed" else spmv64_bytes) + n * (5 * 8 + 2 * 8) + n * (2 * 8 + 2 * 8)
        per_it = profile_traffic(f"pcg_persistent_{precision}_plate2m.md",
                                 "dram_bytes_per_iteration_full_size") if full else None
        return roof(f"k_pcg_persistent<{precision}> (whole PCG solve, one launch)", it_bytes * stx.iterations,
                    stx.solve_seconds, per_it * stx.iterations if per_it else None, bytes_per_iteration=it_bytes,
                    iteration_gbs=it_bytes * stx.iterations / stx.solve_seconds / 1e9)

    jacobi_mixed = {"solve_s": st_jm.solve_seconds, "iterations": st_jm.iterations,
                    "refinements": st_jm.refinements, "true_rel_residual": st_jm.true_rel_residual,
                    "speedup_vs_plain_fp64": st_64.solve_seconds / st_jm.solve_seconds,
                    "roofline": persistent_roof(st_jm, "mixed")}

    # the multigrid hierarchy of this matrix, its cycle and its finest-level smoother sweep
    # (FP32 difference-form operator + FP64 b, D^-1, x in, x out per launch)
    amg = None
    if a.precond == "amg":
        with torch.cuda.stream(stream):
            info = pkg.amg_setup(K)
            tm = pkg.amg_time(K, reps=50)
        sync()
        sweep_bytes = spmv32_bytes + 2 * n * 8
        amg = {"levels": info["levels"], "level_dofs": info["dofs"], "level_nnz": info["nnz"],
               "setup_s": info["setup_seconds"], "vcycle_us": tm["vcycle_s"] * 1e6,
               "cycle": f"V(2,2), {a.amg_smoother} smoothing, FP32 cycle operators, dense coarsest inverse",
               "strength_theta": {"fine": a.amg_theta[0], "coarse": a.amg_theta[1]},
               "tail": {"level": info["tail_level"], "cluster_ctas": info["tail_cluster"]},
               "smoother_roofline": roof("k_amg_sweep_f32 (finest-level smoothing step)", sweep_bytes,
                                         tm["sweep_s"],
                                         profile_traffic("amg_sweep_f32_plate2m.md") if full else None)}
        roofline = amg["smoother_roofline"]
    elif a.precond == "jacobi":
        roofline = persistent_roof(st, a.precision)
    else:
        roofline = roof32

    # accuracy of the headline solution against FP64 Jacobi-PCG under the reference's rule, and
    # the stress concentration factor at the hole (element stresses on the GPU)
    sync()
    x_rel = float(torch.linalg.vector_norm(d_x - x_ref) / torch.linalg.vector_norm(x_ref))
    strs = pkg.compute_element_stresses(ctx, d_x.cpu().numpy(), 1.0, 0.3)
    scf, scf_elem = pkg.scf_at_hole(strs, 1.0)

    dtype = {"amg": "f64 (CG) + f32 (cycle matrix values)", "jacobi": "f64", "learned": "f32+f64+bf16"}
    line = {
        "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": dtype[a.precond] if a.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": f"{a.workload}: {desc}, {n} DOFs, {nnz} nnz, E=1 nu=0.3 plane stress t=1, "
                               "traction (1,0) on x=10, u_x=0 on x=0, u_y=0 on y=0",
                   "step": f"pattern + assembly + Dirichlet + {a.precond} preconditioner setup + PCG to "
                           "rtol 1e-10 on the FP64 true residual",
                   "preconditioner": a.precond, "precision": a.precision, "dofs": n, "nnz": nnz,
                   "l2": f"inputs larger than L2 (FP64 matrix values {nnz * 8 / 1e6:.0f} MB)",
                   "parallelism": f"replicas x{a.gpus}"},
        "time_to_solve_s": t_step, "iterations": st.iterations, "refinements": st.refinements,
        "true_rel_residual": st.true_rel_residual, "solve_s": st.solve_seconds,
        "plain_fp64": {"solve_s": st_64.solve_seconds, "iterations": st_64.iterations,
                       "true_rel_residual": st_64.true_rel_residual,
                       "speedup_of_headline_solve": st_64.solve_seconds / st.solve_seconds,
                       "speedup_of_headline_step": st_64.solve_seconds / t_step},
        "jacobi_mixed": jacobi_mixed,
        "learned_mixed": learned,
        "amg": amg,
        "reference_rule_iterations": st_ref.iterations, "reference_rule_solve_s": st_ref.solve_seconds,
        "x_rel_vs_reference_rule_fp64": x_rel,
        "scf": {"value": scf, "element": scf_elem, "analytic_infinite_plate": 3.0},
        "roofline": roofline,
        "spmv_fp64": roof64,
        "spmv_mixed": roof32,
        "gpu_launches": int(launches),
        "clocks": clk,
    }

    # e2e: through the C ABI with pinned host buffers
    if not a.no_e2e:
        def pinned(arr):
            t = torch.empty(arr.shape, dtype={np.float64: torch.float64, np.int32: torch.int32}[arr.dtype.type],
                            pin_memory=True)
            v = t.numpy()
            v[...] = arr
            return v
        hmesh = pkg.plate.Mesh(xy=pinned(mesh.xy), triangles=pinned(mesh.triangles),
                               boundary_edges=mesh.boundary_edges)
        h_dofs, h_vals, h_b0 = pinned(dofs), pinned(vals), pinned(b0)
        h_b = pinned(b0)
        h_x = pinned(np.zeros(n))
        ectx = pkg.Context(dev)
        ectx.check(ectx.L.cstg_amg_set_smoother(ectx.h, smoother_code))
        ectx.check(ectx.L.cstg_amg_set_strength(ectx.h, *a.amg_theta))

        def e2e_step():
            K2 = pkg.build_stiffness_pattern(hmesh, ctx=ectx)
            pkg.assemble_stiffness(hmesh, D, 1.0, K2)
            np.copyto(h_b, h_b0)
            pkg.apply_dirichlet((h_dofs, h_vals), K2, h_b)
            s2 = pkg.CgJacobiSolver(opts)
            s2.setup(K2)
            if a.precond == "learned":
                pkg.learned.setup(K2, l_weights, l_mat)
            last["e2e"] = s2.solve(h_b, h_x)

        def wall_start():
            return time.perf_counter()

        def wall_stop(t0):
            return time.perf_counter() - t0

        el2 = timed_region(e2e_step, a.steps, a.warmup, dist, wall_start, wall_stop, sync)
        el2 = dist.max(el2, device=f"cuda:{dev}")
        h2d = mesh.xy.nbytes + mesh.triangles.nbytes + dofs.nbytes + vals.nbytes + 2 * b0.nbytes
        d2h = b0.nbytes + h_x.nbytes
        line["e2e"] = {"value": a.gpus * n / (el2 / a.steps), "unit": "DOF/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h), "ms_per_step": el2 / a.steps * 1e3,
                       "path": "C ABI, host pinned buffers (cstg_set_mesh .. cstg_pcg_solve)"}
        ectx.close()

    if dist.rank == 0 and not a.no_cpu_baseline and a.gpus == 1:
        iters_full = st_ref.iterations
        s = cpu_sample(mesh, dofs, vals, a.cpu_sample_iters)
        line["cpu_baseline"] = cpu_baseline_entry(s, n, iters_full, a.cpu_sample_iters)
    ctx.close()
    if dist.rank == 0:
        print(json.dumps(line))
    dist.close()
    return 0


def main():
    a = parse()
    dist = Dist()
    if a.impl == "reference":
        return run_reference(a, dist)
    return run_ours(a, dist)


if __name__ == "__main__":
    sys.exit(main())
