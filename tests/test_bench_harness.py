"""bench.py's multi-rank plumbing on CPU: world size 2 over gloo (127.0.0.1), replicas with
barrier + max-over-ranks timing and no data-path collective; clock parsing."""
import json
import os
import socket
import subprocess
import sys

from conftest import REPO

WORKER = r"""
import os, sys, time, json
sys.path.insert(0, REPO)
import bench
d = bench.Dist()
d.init("gloo")
calls = []
def step():
    calls.append(1)
    time.sleep(0.01 * (d.rank + 1))     # rank 1 is slower: the max must be rank 1's time
t = bench.timed_region(step, 5, 3, d, lambda: time.perf_counter(),
                       lambda t0: time.perf_counter() - t0, lambda: None)
m = d.max(t)
print(json.dumps({"rank": d.rank, "own": t, "max": m, "calls": len(calls)}))
d.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_replica_timing():
    port = _free_port()
    code = "REPO = %r\n" % REPO + WORKER
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    outs.sort(key=lambda x: x["rank"])
    assert all(o["calls"] == 8 for o in outs)
    assert outs[0]["max"] == outs[1]["max"] == max(o["own"] for o in outs)
    assert outs[1]["own"] >= 5 * 0.02 * 0.9


def test_clock_parsing():
    sys.path.insert(0, REPO)
    import bench
    txt = ("1965, 1965, 700.1, Not Active, Not Active, Not Active, Not Active\n"
           "1800, 1965, 990.2, Not Active, Not Active, Not Active, Active\n"
           "1900, 1965, 995.0, Not Active, Not Active, Not Active, Active\n")
    c = bench.parse_clock_csv(txt)
    assert c["sm_mhz"] == 1900 and c["sm_max_mhz"] == 1965 and c["reasons"] == ["sw_power_cap"]


def test_reference_arm_line():
    """`bench.py --impl reference` (the reference's serial core on the host, one bounded sample of
    the 2M-DOF workload per step) prints one JSON line with the contract's keys, flags the
    extrapolation to the iteration count of the reference's own full run, and its figures agree
    with one another: value = DOFs / time-to-solve, ms_per_step = the sample that ran, no
    host-device bytes."""
    import pytest
    import oracle
    if not oracle.RefCore.available():
        pytest.skip("the reference core (oracle/_ref) is not built")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 1 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["extrapolated"] is True and d["sample_iters"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] == 1 and cb["value"] == d["value"]
    n_dofs = 2_000_244
    assert abs(d["value"] * d["time_to_solve_s"] - n_dofs) < 1e-6 * n_dofs
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0 == d["e2e"]["d2h_bytes_per_step"]
    # the sample that ran (setup + sample_iters iterations) is far shorter than the extrapolated solve
    assert 0 < d["ms_per_step"] < 0.1 * d["time_to_solve_s"] * 1e3
