"""add_traction on the GPU (bc.cpp:190-253) against the reference's loads.

Bars: constant traction bit-identical to the reference (golden fixtures of the reference's own
add_traction on its Kirsch meshes, and the host path on the plates); the analytical Kirsch
traction (kirsch.cpp:40-45) within relative 1e-12 of an FP64 evaluation of the same formula
(CUDA's sin / cos / atan2 are not the host library's); an edge that is not a boundary edge is
rejected with f untouched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_device_traction_matches_reference_bits(pkg, gpu_lib, golden, name):
    g = golden(name)
    mesh = g.mesh(pkg)
    K = pkg.build_stiffness_pattern(mesh)
    f = _dev(np.zeros(mesh.num_dofs))
    pkg.add_traction(K, mesh.boundary_edges["right"], 0.01, 100e6, 0.0, f)
    assert np.array_equal(f.cpu().numpy(), g["stress_f"])
    K.ctx.close()


def test_device_traction_matches_host_path_on_plates(pkg, gpu_lib):
    m = pkg.plate.quarter_plate(37, 90, a=1.3)
    K = pkg.build_stiffness_pattern(m)
    fh = np.zeros(m.num_dofs)
    fd = _dev(np.zeros(m.num_dofs))
    for grp, tx, ty in [("right", 1.0, 0.5), ("top", -0.25, 2.0), ("hole", 0.3, 0.1)]:
        pkg.add_traction(K, m.boundary_edges[grp], 0.7, tx, ty, fh)
        pkg.add_traction(K, m.boundary_edges[grp], 0.7, tx, ty, fd)  # accumulates like the host
    assert np.array_equal(fd.cpu().numpy(), fh)
    K.ctx.close()


def _kirsch_loads(mesh, edges, t, a, s):
    """FP64 restatement of bc.cpp:190-253 with the Kirsch traction (kirsch.cpp:7-45)."""
    xy = mesh.xy.reshape(-1, 2)
    tri = mesh.triangles.reshape(-1, 3)
    f = np.zeros(mesh.num_dofs)
    g = 1.0 / np.sqrt(3.0)
    for a_, b_ in np.asarray(edges).reshape(-1, 2):
        cand = [tt for tt in tri if a_ in tt and b_ in tt]
        c = [v for v in cand[0] if v not in (a_, b_)][0]
        (xa, ya), (xb, yb) = xy[a_], xy[b_]
        ln = np.hypot(xb - xa, yb - ya)
        nx, ny = (yb - ya) / ln, -(xb - xa) / ln
        if nx * (xy[c, 0] - xa) + ny * (xy[c, 1] - ya) > 0:
            nx, ny = -nx, -ny
        for q in (-g, g):
            Na, Nb = 0.5 * (1 - q), 0.5 * (1 + q)
            x, y = Na * xa + Nb * xb, Na * ya + Nb * yb
            r, th = np.hypot(x, y), np.arctan2(y, x)
            q2 = a * a / (r * r)
            q4 = q2 * q2
            c2, s2 = np.cos(2 * th), np.sin(2 * th)
            rr = 0.5 * s * (1 - q2) + 0.5 * s * (1 - 4 * q2 + 3 * q4) * c2
            tt_ = 0.5 * s * (1 + q2) - 0.5 * s * (1 + 3 * q4) * c2
            rt = -0.5 * s * (1 + 2 * q2 - 3 * q4) * s2
            cc, sn = np.cos(th), np.sin(th)
            sxx = rr * cc * cc + tt_ * sn * sn - 2 * rt * sn * cc
            syy = rr * sn * sn + tt_ * cc * cc + 2 * rt * sn * cc
            sxy = (rr - tt_) * sn * cc + rt * (cc * cc - sn * sn)
            w = t * 0.5 * ln
            for node, N in ((a_, Na), (b_, Nb)):
                f[2 * node] += w * N * (sxx * nx + sxy * ny)
                f[2 * node + 1] += w * N * (sxy * nx + syy * ny)
    return f


def test_device_kirsch_traction(pkg, gpu_lib):
    m = pkg.plate.quarter_plate(12, 24)
    K = pkg.build_stiffness_pattern(m)
    f = _dev(np.zeros(m.num_dofs))
    edges = np.concatenate([m.boundary_edges["right"], m.boundary_edges["top"]])
    pkg.add_kirsch_traction(K, edges, 1.0, 1.0, 1.0, f)
    ref = _kirsch_loads(m, edges, 1.0, 1.0, 1.0)
    assert np.linalg.norm(f.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
    K.ctx.close()


def test_device_traction_rejects_interior_edge(pkg, gpu_lib):
    m = pkg.plate.quarter_plate(6, 8)
    K = pkg.build_stiffness_pattern(m)
    tri = m.triangles.reshape(-1, 3)
    interior = np.array([[tri[0][0], tri[0][2]]], dtype=np.int32)  # the quad diagonal: two triangles
    edges = np.concatenate([m.boundary_edges["right"], interior])
    f = _dev(np.zeros(m.num_dofs))
    with pytest.raises(pkg.CstgError, match="exactly one triangle"):
        pkg.add_traction(K, edges, 1.0, 1.0, 0.0, f)
    assert float(f.abs().sum()) == 0.0
    K.ctx.close()


def test_host_pointer_traction_paths(pkg, gpu_lib):
    """cstg_add_traction with a host f: after cstg_build_pattern it runs on the GPU (f up, the
    pattern's node incidence, f down); before it, on the host from the mesh read back from the
    device. Both give the same bits, accumulating into f; an interior edge is reported with the
    reference's message (the triangle count) and f is left as it was."""
    import ctypes as C
    m = pkg.plate.quarter_plate(23, 52, a=1.1)
    xy = np.ascontiguousarray(m.xy, dtype=np.float64)
    tri = np.ascontiguousarray(m.triangles, dtype=np.int32)
    groups = [("right", 1.0, 0.5), ("top", -0.25, 2.0), ("hole", 0.3, 0.1)]
    out = {}
    for name, build in (("host", False), ("device", True)):
        ctx = pkg.Context(0)
        ctx.check(ctx.L.cstg_set_mesh(ctx.h, m.num_nodes, xy.ctypes.data, m.num_triangles, tri.ctypes.data))
        if build:
            nnz = C.c_int64(0)
            ctx.check(ctx.L.cstg_build_pattern(ctx.h, C.byref(nnz)))
        f = np.full(m.num_dofs, 0.125)
        for grp, tx, ty in groups:
            e = np.ascontiguousarray(m.boundary_edges[grp], dtype=np.int32).reshape(-1)
            ctx.check(ctx.L.cstg_add_traction(ctx.h, e.size // 2, e.ctypes.data, 0.7, tx, ty, f.ctypes.data))
        out[name] = f
        t3 = tri.reshape(-1, 3)
        bad = np.ascontiguousarray(np.concatenate([m.boundary_edges["right"].reshape(-1, 2),
                                                   [[t3[0][0], t3[0][2]]]]), dtype=np.int32).reshape(-1)
        g = f.copy()
        rc = ctx.L.cstg_add_traction(ctx.h, bad.size // 2, bad.ctypes.data, 1.0, 1.0, 0.0, g.ctypes.data)
        assert rc == pkg.native.ERR_MESH
        assert "is adjacent to 2 triangles" in ctx.L.cstg_last_error(ctx.h).decode()
        assert np.array_equal(g, f)
        ctx.close()
    assert np.array_equal(out["host"], out["device"])
