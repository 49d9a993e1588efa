"""The host-side .msh 4.1 reader (csrc/mesh_io.cu: plain host C++ behind the C ABI) built with
AddressSanitizer and UndefinedBehaviorSanitizer (g++ -fsanitize=address,undefined, every report
fatal) and fed a valid file and malformed ones: truncations, corrupted counts, bad tokens, a
triangle on a missing node, wrong format headers, NUL bytes, an overlong line and seeded byte
corruptions. Each run must end in "ok" or a clean error status with no sanitizer report, and a
mesh the reader accepts must keep its indices inside the nodes. (The GPU code has no sanitizer on
this pool; the host parser, which reads untrusted files, is checked here.)"""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(REPO, "mpi-cst-fem-solver_b200", "csrc", "mesh_io.cu")
MAIN = os.path.join(HERE, "sanitize", "read_msh_main.cpp")
ENV = dict(os.environ, ASAN_OPTIONS="allocator_may_return_null=1:detect_leaks=1:abort_on_error=0",
           UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")


@pytest.fixture(scope="module")
def reader(tmp_path_factory):
    gxx = shutil.which("g++") or "/usr/bin/g++"
    if not os.path.exists(gxx):
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("asan") / "read_msh")
    cmd = [gxx, "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           "-fno-omit-frame-pointer", "-x", "c++", SRC, "-x", "c++", MAIN, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "asan" in r.stderr.lower():
        pytest.skip("sanitizer runtime not available: " + r.stderr.strip()[-200:])
    assert r.returncode == 0, r.stderr
    return exe


def _run(exe, path):
    r = subprocess.run([exe, path], capture_output=True, text=True, env=ENV, timeout=120)
    report = "AddressSanitizer" in r.stderr or "runtime error" in r.stderr or "LeakSanitizer" in r.stderr
    assert not report and r.returncode == 0, (path, r.returncode, r.stdout, r.stderr[-2000:])
    return r.stdout.split(None, 3)


@pytest.fixture(scope="module")
def valid(pkg, tmp_path_factory):
    mesh = pkg.plate.quarter_plate(4, 8)
    path = str(tmp_path_factory.mktemp("msh") / "plate.msh")
    pkg.write_gmsh(mesh, path)
    return mesh, path, open(path, "rb").read()


def _variant(tmp_path, name, data):
    p = str(tmp_path / name)
    with open(p, "wb") as f:
        f.write(data)
    return p


def test_valid_file(reader, valid):
    mesh, path, _ = valid
    out = _run(reader, path)
    assert out[0] == "ok", out
    assert int(out[1]) == mesh.num_nodes and int(out[2]) == np.asarray(mesh.triangles).size // 3
    assert int(out[3]) == len(mesh.boundary_edges)  # the boundary edge groups


def test_malformed_files_end_cleanly(reader, valid, tmp_path):
    mesh, _, data = valid
    text = data.decode()
    n = mesh.num_nodes
    must_fail = {
        "empty": b"",
        "binary": data.replace(b"4.1 0 8", b"4.1 1 8"),
        "version": data.replace(b"4.1 0 8", b"2.2 0 8"),
        "huge_count": text.replace(f"$Nodes\n1 {n} 1 {n}", "$Nodes\n1 2147483647 1 2147483647").encode(),
        "negative_count": text.replace(f"$Nodes\n1 {n} 1 {n}", f"$Nodes\n1 -3 1 {n}").encode(),
        "bad_token": text.replace(f"2 1 0 {n}\n", "2 1 0 abc\n").encode(),
        "missing_node": text.replace("$EndElements", "").rstrip().rsplit("\n", 1)[0].encode()
        + f"\n999 1 2 {n + 7}\n$EndElements\n".encode(),
        "no_end_nodes": data.replace(b"$EndNodes", b""),
    }
    for name, d in must_fail.items():
        out = _run(reader, _variant(tmp_path, name + ".msh", d))
        assert out[0] == "err", (name, out)
    others = {"nul_bytes": data[: len(data) // 2] + b"\0" * 64 + data[len(data) // 2:],
              "long_line": data.replace(b"$Nodes", b"$Comments\n" + b"7" * 100000 + b"\n$EndComments\n$Nodes")}
    for k in range(1, 25):  # truncations
        others[f"trunc{k}"] = data[: len(data) * k // 25]
    rng = np.random.default_rng(2026)
    for k in range(40):  # one corrupted byte each, anywhere in the file
        b = bytearray(data)
        i = int(rng.integers(0, len(b)))
        b[i] = int(rng.choice(list(b"0123456789-+.eE \n$abc")))
        others[f"flip{k}"] = bytes(b)
    for name, d in others.items():
        out = _run(reader, _variant(tmp_path, name + ".msh", d))
        assert out[0] in ("ok", "err"), (name, out)
