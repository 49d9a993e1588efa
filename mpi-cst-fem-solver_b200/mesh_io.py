"""Gmsh .msh 4.1 meshes: the library's reader (cstg_read_gmsh, the reference's read_gmsh,
src/mesh_io.cpp) and a writer for generated meshes (plates), so that files feed the GPU path."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .native import CstgError
from .plate import Mesh


def read_gmsh(path: str) -> Mesh:
    """Reads a .msh 4.1 ASCII file: Mesh(xy, triangles, boundary_edges) with `node_tags` and
    `flipped` (triangles turned counter-clockwise) attached. Raises CstgError("path:line: ...")."""
    L = native.load()
    h = C.c_void_p()
    err = C.create_string_buffer(1024)
    rc = L.cstg_read_gmsh(str(path).encode(), C.byref(h), err, len(err))
    if rc:
        raise CstgError(rc, err.value.decode())
    try:
        nn, nt, ng, fl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.cstg_mesh_info(h, C.byref(nn), C.byref(nt), C.byref(ng), C.byref(fl))
        xy = np.zeros(2 * nn.value)
        tri = np.zeros(3 * nt.value, dtype=np.int32)
        tags = np.zeros(nn.value, dtype=np.int64)
        L.cstg_mesh_arrays(h, xy.ctypes.data, tri.ctypes.data, tags.ctypes.data)
        groups = {}
        for g in range(ng.value):
            name = C.create_string_buffer(512)
            ne = C.c_int()
            L.cstg_mesh_group(h, g, name, len(name), C.byref(ne), None)
            e = np.zeros(2 * ne.value, dtype=np.int32)
            L.cstg_mesh_group(h, g, name, len(name), C.byref(ne), e.ctypes.data)
            groups[name.value.decode()] = e.reshape(-1, 2)
    finally:
        L.cstg_mesh_destroy(h)
    m = Mesh(xy=xy, triangles=tri, boundary_edges=groups)
    m.node_tags = tags
    m.flipped = fl.value
    return m


def write_gmsh(mesh: Mesh, path: str) -> None:
    """Writes the mesh as .msh 4.1 ASCII: one surface entity holding the triangles, one curve
    entity (and physical group of the same name) per boundary group; node tags 1..N."""
    xy = np.asarray(mesh.xy).reshape(-1, 2)
    tri = np.asarray(mesh.triangles).reshape(-1, 3)
    names = list(mesh.boundary_edges)
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        f.write(f"$PhysicalNames\n{len(names) + 1}\n")
        for k, nm in enumerate(names):
            f.write(f'1 {k + 1} "{nm}"\n')
        f.write(f'2 {len(names) + 1} "domain"\n$EndPhysicalNames\n')
        lo, hi = xy.min(axis=0).tolist(), xy.max(axis=0).tolist()
        box = f"{lo[0]!r} {lo[1]!r} 0 {hi[0]!r} {hi[1]!r} 0"
        f.write(f"$Entities\n0 {len(names)} 1 0\n")
        for k in range(len(names)):
            f.write(f"{k + 1} {box} 1 {k + 1} 0\n")
        f.write(f"1 {box} 1 {len(names) + 1} 0\n$EndEntities\n")
        n = xy.shape[0]
        f.write(f"$Nodes\n1 {n} 1 {n}\n2 1 0 {n}\n")
        f.write("".join(f"{i + 1}\n" for i in range(n)))
        f.write("".join(f"{x!r} {y!r} 0\n" for x, y in xy.tolist()))
        f.write("$EndNodes\n")
        n_lines = sum(np.asarray(mesh.boundary_edges[nm]).reshape(-1, 2).shape[0] for nm in names)
        f.write(f"$Elements\n{len(names) + 1} {n_lines + tri.shape[0]} 1 {n_lines + tri.shape[0]}\n")
        tag = 1
        for k, nm in enumerate(names):
            e = np.asarray(mesh.boundary_edges[nm]).reshape(-1, 2)
            f.write(f"1 {k + 1} 1 {e.shape[0]}\n")
            for a, b in e:
                f.write(f"{tag} {a + 1} {b + 1}\n")
                tag += 1
        f.write(f"2 1 2 {tri.shape[0]}\n")
        for a, b, c in tri:
            f.write(f"{tag} {a + 1} {b + 1} {c + 1}\n")
            tag += 1
        f.write("$EndElements\n")
