"""Synthetic quarter plates with a circular hole (O-grid CST meshes).

The reference meshes its Kirsch plates with Gmsh (python/mesh_kirsch.py); Gmsh is not part of
this build, so the plates used by the benchmark and the size-independent tests are generated
here. A plate is the square [0, L]^2 minus the disc r < a, meshed by rays:

* node (i, j), i = 0..n_r along ray j = 0..n_theta, theta_j = (pi/2) j / n_theta;
* the ray runs from (a cos t, a sin t) to the square boundary (x = L while cos t > sin t,
  y = L while sin t > cos t, the corner (L, L) at j = n_theta / 2, so n_theta must be even);
* radial spacing is geometric with ratio q = grading^(40 / n_r) per cell, which keeps the total
  last/first ratio of a 40-cell mesh graded by `grading` (a constant 1.05 per cell would
  degenerate at large n_r);
* node index j * (n_r + 1) + i (ray-major: matrix bandwidth n_r + 1);
* each quad (i, j) is split into the counter-clockwise triangles (n00, n10, n11), (n00, n11, n01);
* boundary line groups carry the reference's names: hole, left_sym (x = 0), bottom_sym (y = 0),
  right (x = L), top (y = L).

The mesh arrays follow the reference's `Mesh` (include/cstfem/mesh.hpp:19-30): xy is
(x0, y0, x1, y1, ...) float64, triangles is int32 3 per element, counter-clockwise, 0-based,
and boundary_edges maps a group name to int32 (n_edges, 2) node pairs.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


def _count(a) -> int:
    return int(a.numel()) if hasattr(a, "numel") else int(a.size)


@dataclasses.dataclass
class Mesh:
    xy: np.ndarray  # float64 [2 * n_nodes]
    triangles: np.ndarray  # int32 [3 * n_tri]
    boundary_edges: dict  # name -> int32 [n_edges, 2]

    # (numpy arrays or CUDA tensors: both have numel via .size / .numel())
    @property
    def num_nodes(self) -> int:
        return _count(self.xy) // 2

    @property
    def num_triangles(self) -> int:
        return _count(self.triangles) // 3

    @property
    def num_dofs(self) -> int:
        return 2 * self.num_nodes


def radial_fractions(n_r: int, grading: float = 1.05) -> np.ndarray:
    """t_i in [0, 1], geometric with per-cell ratio grading**(40/n_r); t_0 = 0, t_{n_r} = 1."""
    q = grading ** (40.0 / n_r)
    i = np.arange(n_r + 1, dtype=np.float64)
    if q == 1.0:
        t = i / n_r
    else:
        t = (q ** i - 1.0) / (q ** n_r - 1.0)
    t[0] = 0.0
    t[-1] = 1.0
    return t


def quarter_plate(n_r: int, n_theta: int, a: float = 1.0, L: float = 10.0,
                  grading: float = 1.05) -> Mesh:
    """O-grid quarter plate [0, L]^2 minus the disc r < a; see the module docstring."""
    if n_r < 1 or n_theta < 2 or n_theta % 2:
        raise ValueError(f"quarter_plate: need n_r >= 1 and an even n_theta >= 2, got {n_r}, {n_theta}")
    if not (0.0 < a < L):
        raise ValueError(f"quarter_plate: need 0 < a < L, got a={a}, L={L}")
    j = np.arange(n_theta + 1)
    th = (math.pi / 2.0) * j / n_theta
    c, s = np.cos(th), np.sin(th)
    c[0], s[0] = 1.0, 0.0
    c[-1], s[-1] = 0.0, 1.0
    jc = n_theta // 2
    inner = np.stack([a * c, a * s], axis=1)
    outer = np.empty_like(inner)
    lo, hi = j < jc, j > jc
    outer[lo, 0] = L
    outer[lo, 1] = L * s[lo] / c[lo]
    outer[hi, 0] = L * c[hi] / s[hi]
    outer[hi, 1] = L
    outer[jc] = (L, L)
    t = radial_fractions(n_r, grading)
    # [n_theta + 1, n_r + 1, 2], ray-major
    pts = inner[:, None, :] + t[None, :, None] * (outer - inner)[:, None, :]
    pts[:, 0, :] = inner
    pts[:, -1, :] = outer
    xy = np.ascontiguousarray(pts.reshape(-1), dtype=np.float64)

    nr1 = n_r + 1
    jj, ii = np.meshgrid(np.arange(n_theta), np.arange(n_r), indexing="ij")
    n00 = (jj * nr1 + ii).reshape(-1)
    n10 = n00 + 1
    n01 = n00 + nr1
    n11 = n01 + 1
    tri = np.empty((n00.size, 2, 3), dtype=np.int32)
    tri[:, 0] = np.stack([n00, n10, n11], axis=1)
    tri[:, 1] = np.stack([n00, n11, n01], axis=1)
    triangles = np.ascontiguousarray(tri.reshape(-1))

    def chain(nodes):
        nodes = np.asarray(nodes, dtype=np.int32)
        return np.ascontiguousarray(np.stack([nodes[:-1], nodes[1:]], axis=1))

    i_all = np.arange(nr1)
    groups = {
        "hole": chain(np.arange(n_theta + 1) * nr1),
        "left_sym": chain(n_theta * nr1 + i_all),
        "bottom_sym": chain(i_all),
        "right": chain(np.arange(jc + 1) * nr1 + n_r),
        "top": chain(np.arange(jc, n_theta + 1) * nr1 + n_r),
    }
    return Mesh(xy=xy, triangles=triangles, boundary_edges=groups)


def group_nodes(mesh: Mesh, group: str) -> np.ndarray:
    """Sorted unique nodes of a boundary group."""
    return np.unique(mesh.boundary_edges[group].reshape(-1))


def symmetry_dirichlet(mesh: Mesh):
    """u_x = 0 on left_sym, u_y = 0 on bottom_sym as sorted (dofs int32, values float64), the
    set the reference's `bc.dirichlet = left_sym:ux=0 ; bottom_sym:uy=0` produces."""
    d = np.concatenate([2 * group_nodes(mesh, "left_sym"), 2 * group_nodes(mesh, "bottom_sym") + 1])
    d = np.unique(d).astype(np.int32)
    return d, np.zeros(d.size, dtype=np.float64)


# The four load cases of the batched plates: (group, tx, ty) lists.
LOAD_CASES = {
    "tension_x": [("right", 1.0, 0.0)],
    "tension_y": [("top", 0.0, 1.0)],
    "shear": [("right", 0.0, 1.0), ("top", 1.0, 0.0)],
    "biaxial": [("right", 1.0, 0.0), ("top", 0.0, 1.0)],
}


@dataclasses.dataclass
class PlateSpec:
    """One plate of a seeded batch (the uneven-size batch workload)."""
    n_r: int
    n_theta: int
    a: float
    E: float
    nu: float
    plane_strain: bool


def random_batch(count: int = 64, seed: int = 2026, n_r_range=(20, 200)) -> list:
    """Seeded plates: a ~ U(0.5, 2), n_r ~ U{lo..hi}, n_theta = 2 n_r, E ~ U(0.5, 2),
    nu ~ U(0.2, 0.45), plane strain with probability 1/2."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n_r = int(rng.integers(n_r_range[0], n_r_range[1] + 1))
        out.append(PlateSpec(n_r=n_r, n_theta=2 * n_r, a=float(rng.uniform(0.5, 2.0)),
                             E=float(rng.uniform(0.5, 2.0)), nu=float(rng.uniform(0.2, 0.45)),
                             plane_strain=bool(rng.integers(0, 2))))
    return out
