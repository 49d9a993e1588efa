"""The reference-side GPU backend (tests/binding/gpu_backend.hpp: GpuStiffness, GpuOperator,
CgJacobiGpuSolver over the C ABI) compiled against the reference's own headers and linked with
its serial core: the reference's PCG test cases and its serial driver flow on the Kirsch L0 mesh
run through the GPU (tests/binding/test_gpu_binding.cpp). The program is built where the
reference's headers exist (`make -C tests/binding`, also run by __graft_entry__.build()) and
travels with the library."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "binding", "_build", "test_gpu_binding")


def test_reference_binding_runs_the_reference_cases_on_the_gpu(pkg, gpu_lib, golden, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("binding test program not built (needs the reference's headers: make -C tests/binding)")
    msh = str(tmp_path / "kirsch_L0.msh")
    pkg.write_gmsh(golden("kirsch_L0").mesh(pkg), msh)  # the reference reader's mesh, rewritten
    out = subprocess.run([BIN, msh], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert " 0 failed" in out.stdout
