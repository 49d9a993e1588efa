"""Host-side front end: the .msh 4.1 reader (against the reference's reader through the golden
fixtures and, when the reference checkout is present, its own files), the writer, and the
case-file parser (the reference's format and error rules). CPU only."""
import os
import re

import numpy as np
import pytest

from oracle import REF_DIR as REF  # the reference checkout (beside the repository, or $CSTFEM_REF)
GROUPS = ("hole", "left_sym", "bottom_sym", "right", "top")


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_read_gmsh_matches_reference_reader(pkg, gpu_lib, golden, name):
    path = os.path.join(REF, "tests", "data", name + ".msh")
    if not os.path.exists(path):
        pytest.skip("reference mesh files not present")
    g = golden(name)
    m = pkg.read_gmsh(path)
    assert np.array_equal(m.xy, g["xy"]) and np.array_equal(m.triangles, g["tri"])
    assert m.flipped == int(g["flipped"])
    for grp in GROUPS:
        assert np.array_equal(m.boundary_edges[grp].reshape(-1), g["group_" + grp].reshape(-1))


def test_write_read_round_trip(pkg, gpu_lib, golden, tmp_path):
    for mesh in (pkg.plate.quarter_plate(9, 14, a=0.7), golden("kirsch_L0").mesh(pkg)):
        p = str(tmp_path / "m.msh")
        pkg.write_gmsh(mesh, p)
        m = pkg.read_gmsh(p)
        assert np.array_equal(m.xy, mesh.xy) and np.array_equal(m.triangles, mesh.triangles)
        assert m.flipped == 0 and np.array_equal(m.node_tags, np.arange(1, mesh.num_nodes + 1))
        for grp, e in mesh.boundary_edges.items():
            assert np.array_equal(m.boundary_edges[grp].reshape(-1), np.asarray(e).reshape(-1))


def test_read_gmsh_flips_clockwise_triangles(pkg, gpu_lib, tmp_path):
    mesh = pkg.plate.quarter_plate(3, 4)
    tri = mesh.triangles.reshape(-1, 3).copy()
    tri[::2] = tri[::2, [0, 2, 1]]  # every other triangle clockwise
    p = str(tmp_path / "cw.msh")
    pkg.write_gmsh(pkg.plate.Mesh(xy=mesh.xy, triangles=tri.reshape(-1), boundary_edges=mesh.boundary_edges), p)
    m = pkg.read_gmsh(p)
    assert m.flipped == (tri.shape[0] + 1) // 2
    assert np.array_equal(m.triangles, mesh.triangles)


def _bad_first_element(s):
    lines = s.split("\n")
    k = lines.index("$Elements") + 3  # header, first block header, first element
    lines[k] = " ".join(lines[k].split()[:-1] + ["99999"])
    return "\n".join(lines)


@pytest.mark.parametrize("edit,msg", [
    (lambda s: s.replace("4.1 0 8", "2.2 0 8"), "unsupported .msh version '2.2'"),
    (lambda s: s.replace("4.1 0 8", "4.1 1 8"), "binary .msh files are not supported"),
    (lambda s: s.replace("$PhysicalNames", "$Foo", 1).replace("$EndPhysicalNames", "$EndFoo", 1),
     "missing $PhysicalNames section"),
    (lambda s: _bad_first_element(s), "unknown node tag 99999"),
])
def test_read_gmsh_errors(pkg, gpu_lib, tmp_path, edit, msg):
    mesh = pkg.plate.quarter_plate(2, 2)
    p = str(tmp_path / "bad.msh")
    pkg.write_gmsh(mesh, p)
    s = open(p).read()
    s2 = edit(s)
    assert s2 != s
    open(p, "w").write(s2)
    with pytest.raises(pkg.CstgError, match=re.escape(msg)):
        pkg.read_gmsh(p)
    try:
        pkg.read_gmsh(p)
    except pkg.CstgError as e:
        assert str(e).startswith(p + ":")


def test_case_file_parsing(pkg):
    from importlib import import_module
    case = import_module("mpi-cst-fem-solver_b200.case")
    text = ("# comment\nmesh = m.msh   # trailing\nplane = plane_stress\nE = 210e9\nnu = 0.3\n"
            "thickness = 0.01\nsolver = gpu_cg_mixed\nrtol = 1e-10\nmax_iter = 5000\n"
            "bc.dirichlet = left_sym:ux=0 ; bottom_sym:uy=0\nbc.traction = right:tx=1e6,ty=0\nfoo = 1\n")
    c = case.CaseFile.parse(text, "t.case")
    s = case.read_case_settings(c)
    assert s["mesh"] == "m.msh" and s["E"] == 210e9 and s["max_iter"] == 5000 and s["solver"] == "gpu_cg_mixed"
    import io
    err = io.StringIO()
    assert c.warn_unknown_keys(case.KNOWN_KEYS, err) == 1 and "t.case:12: unknown key 'foo'" in err.getvalue()
    assert case.parse_dirichlet("left_sym:ux=0 ; bottom_sym:uy=0") == [
        {"group": "left_sym", "ux": 0.0}, {"group": "bottom_sym", "uy": 0.0}]
    assert case.parse_traction("right:tx=2") == [{"group": "right", "tx": 2.0, "ty": 0.0}]
    bad = [("a = 1\na = 2\n", "duplicate key 'a' (first defined on line 1)"),
           ("a b = 1\n", "key 'a b' contains whitespace"), ("novalue\n", "expected 'key = value'")]
    for t, m in bad:
        with pytest.raises(case.CaseError, match=re.escape(m)):
            case.CaseFile.parse(t, "x")
    with pytest.raises(case.CaseError, match="unknown component 'uz'"):
        case.parse_dirichlet("g:uz=0")
    with pytest.raises(case.CaseError, match="'tx' given twice"):
        case.parse_traction("g:tx=1,tx=2")
    with pytest.raises(case.CaseError, match="not a number"):
        case.parse_traction("g:tx=abc")
    with pytest.raises(case.CaseError, match="petsc is not available"):
        case.read_case_settings(case.CaseFile.parse(text.replace("gpu_cg_mixed", "petsc")))


def test_reference_case_files_parse(pkg):
    from importlib import import_module
    case = import_module("mpi-cst-fem-solver_b200.case")
    d = os.path.join(REF, "cases")
    if not os.path.isdir(d):
        pytest.skip("reference case files not present")
    for f in sorted(os.listdir(d)):
        if f.startswith("kirsch"):
            s = case.read_case_settings(case.CaseFile.load(os.path.join(d, f)))
            assert s["solver"] == "cg_jacobi" and s["plane_name"] in ("plane_stress", "plane_strain")
