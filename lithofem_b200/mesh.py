"""Synthetic conformal tetrahedral meshes of Bloch-periodic layer stacks.

The reference meshes its stacks with gmsh (src/lithofem/meshgen.py:365-513),
which is not available here.  This module builds structured conformal meshes
of the same geometries: a tensor grid whose lines sit on every material
interface (layer z-breakpoints, PML interfaces, frustum side walls), each hex
split into the 6 Kuhn (Freudenthal) tetrahedra, which tile any tensor grid
conformally.  Sloped frustum walls are produced by moving grid nodes with z so
that wall nodes stay on the wall plane; the topology is unchanged, so the mesh
stays conformal.  Lateral periodicity is vertex identification
(node i = nx is node 0), as in the reference's ``$Periodic`` mesh
(meshgen.py:485-506); geometry keeps the unwrapped coordinates, the way the
reference's periodic mesh carries per-element nodes (asm_data.inc:149-151).

Region/attribute convention (src/lithofem/config.py:689-735): attribute =
1-based index into the region list, enumerated slab-major, within a slab the
background first and then each frustum spanning the slab; the bottom and top
PML slabs come last, in that order.
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Frustum:
    """Rectangular frustum: base [x0,x1] x [y0,y1] at z0, height h (may be < 0).

    ``alpha`` is the side-wall angle in degrees; alpha < 90 narrows the
    cross-section away from the base.  A rectangle spanning a whole periodic
    period in y (y0 = 0, y1 = Ly) is a line of a grating.
    """

    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    h: float
    alpha: float
    eps: complex

    @property
    def z_lo(self) -> float:
        return min(self.z0, self.z0 + self.h)

    @property
    def z_hi(self) -> float:
        return max(self.z0, self.z0 + self.h)

    def inset(self, z: np.ndarray) -> np.ndarray:
        """Lateral inset of the walls at height z (0 at the base)."""
        z = np.asarray(z, dtype=float)
        t = 1.0 / math.tan(math.radians(self.alpha)) if self.alpha != 90 else 0.0
        dz = np.clip(np.abs(z - self.z0), 0.0, abs(self.h))
        return dz * t


@dataclass
class Stack:
    """Bloch-periodic layer stack (the part of the reference Model the path reads)."""

    lx: float
    ly: float
    z_min: float
    z_max: float
    wavelength: float
    background_eps: complex = 1.0 + 0j
    layers: list[tuple[float, float, complex]] = field(default_factory=list)
    frustums: list[Frustum] = field(default_factory=list)
    pml_thickness_wavelengths: float = 1.0
    pml_order: float = 2.0
    pml_target: float = 1e-8

    @property
    def k0(self) -> float:
        return 2.0 * math.pi / self.wavelength

    @property
    def pml_thick(self) -> float:
        return self.pml_thickness_wavelengths * self.wavelength

    @property
    def slabs(self) -> list[float]:
        """z breakpoints of the stack: the domain bounds, layer faces and
        frustum base / top planes inside the domain, as the reference's
        z_breakpoints (src/lithofem/geometry.py:221-244), so that every
        frustum spans whole slabs."""
        zs = {self.z_min, self.z_max}
        for z0, z1, _ in self.layers:
            zs.update((z0, z1))
        for f in self.frustums:
            zs.update((f.z_lo, f.z_hi))
        return sorted(z for z in zs if self.z_min <= z <= self.z_max)

    def eps_bg_of_slab(self, i: int) -> complex:
        s = self.slabs
        zc = 0.5 * (s[i] + s[i + 1])
        eps = self.background_eps
        for z0, z1, e in self.layers:
            if z0 <= zc <= z1:
                eps = e
        return complex(eps)

    def regions(self) -> list[dict]:
        """Region table in attribute order (config.py:700-735)."""
        out = []
        s = self.slabs
        for i in range(len(s) - 1):
            zc = 0.5 * (s[i] + s[i + 1])
            out.append({"slab": i, "z": (s[i], s[i + 1]), "kind": "background",
                        "eps": self.eps_bg_of_slab(i)})
            for j, f in enumerate(self.frustums):
                if f.z_lo <= zc <= f.z_hi:
                    out.append({"slab": i, "z": (s[i], s[i + 1]), "kind": "frustum",
                                "frustum": j, "eps": complex(f.eps)})
        n_slab = len(s) - 1
        t = self.pml_thick
        out.append({"slab": -1, "z": (self.z_min - t, self.z_min), "kind": "pml_bottom",
                    "eps": self.eps_bg_of_slab(0)})
        out.append({"slab": n_slab, "z": (self.z_max, self.z_max + t), "kind": "pml_top",
                    "eps": self.eps_bg_of_slab(n_slab - 1)})
        return out


@dataclass
class TetMesh:
    """Conformal periodic tetrahedral mesh.

    ``tv`` (ne, 4) topological vertex ids after periodic identification;
    ``xv`` (ne, 4, 3) the element's own (unwrapped) vertex coordinates;
    ``attr`` (ne,) 1-based region attribute; ``nv`` topological vertex count.
    """

    tv: np.ndarray
    xv: np.ndarray
    attr: np.ndarray
    nv: int
    grid: tuple[int, int, int] = (0, 0, 0)

    @property
    def ne(self) -> int:
        return int(self.tv.shape[0])


def _axis_nodes(breaks: list[float], h: float, min_cells: int = 1) -> np.ndarray:
    breaks = sorted(set(float(b) for b in breaks))
    nodes = [breaks[0]]
    for a, b in zip(breaks[:-1], breaks[1:]):
        n = max(min_cells, int(math.ceil((b - a) / h - 1e-9)))
        nodes.extend(a + (b - a) * np.arange(1, n + 1) / n)
    return np.array(nodes)


# Kuhn subdivision of the unit cube: one tet per axis permutation, path
# 000 -> e_a -> e_a + e_b -> 111.
_KUHN = []
for _perm in itertools.permutations(range(3)):
    _c = [np.zeros(3, dtype=int)]
    for _ax in _perm:
        _n = _c[-1].copy()
        _n[_ax] = 1
        _c.append(_n)
    _KUHN.append(np.array(_c))
_KUHN = np.array(_KUHN)  # (6, 4, 3) corner offsets


def build_mesh(stack: Stack, h: float, h_xy: float | None = None,
               min_lateral_cells: int = 3) -> TetMesh:
    """Mesh ``stack`` (domain plus both PML slabs) with target edge length h."""
    hx = h_xy if h_xy is not None else h
    t = stack.pml_thick
    xb = [0.0, stack.lx]
    yb = [0.0, stack.ly]
    zb = [stack.z_min - t, stack.z_min, stack.z_max, stack.z_max + t] + stack.slabs
    for f in stack.frustums:
        for x in (f.x0, f.x1):
            if 0.0 < x < stack.lx:
                xb.append(x)
        for y in (f.y0, f.y1):
            if 0.0 < y < stack.ly:
                yb.append(y)
        zb += [f.z_lo, f.z_hi]
    xn = _axis_nodes(xb, hx)
    yn = _axis_nodes(yb, hx)
    zn = _axis_nodes(zb, h)
    nx, ny, nz = len(xn) - 1, len(yn) - 1, len(zn) - 1
    if nx < min_lateral_cells or ny < min_lateral_cells:
        xn = _axis_nodes(xb, min(hx, stack.lx / min_lateral_cells))
        yn = _axis_nodes(yb, min(hx, stack.ly / min_lateral_cells))
        nx, ny = len(xn) - 1, len(yn) - 1

    # node coordinates (nx+1, ny+1, nz+1, 3), then side-wall node motion
    X, Y, Z = np.meshgrid(xn, yn, zn, indexing="ij")
    P = np.stack([X, Y, Z], axis=-1).copy()
    for f in stack.frustums:
        if f.alpha == 90:
            continue
        for axis, (lo, hi), nodes, L, allb in ((0, (f.x0, f.x1), xn, stack.lx, xb),
                                               (1, (f.y0, f.y1), yn, stack.ly, yb)):
            brk = np.array(sorted(set(float(b) for b in allb)))
            for k, zk in enumerate(zn):
                if not (f.z_lo - 1e-12 <= zk <= f.z_hi + 1e-12):
                    continue
                d = float(f.inset(zk))
                if d == 0.0:
                    continue
                tgt = brk.copy()
                if lo > 0.0:
                    tgt[np.isclose(brk, lo)] = lo + d
                if hi < L:
                    tgt[np.isclose(brk, hi)] = hi - d
                src = np.interp(nodes, brk, tgt)
                if axis == 0:
                    P[:, :, k, 0] = src[:, None]
                else:
                    P[:, :, k, 1] = src[None, :]

    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cubes = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)  # (nc, 3)
    corner = cubes[:, None, None, :] + _KUHN[None, :, :, :]          # (nc, 6, 4, 3)
    corner = corner.reshape(-1, 4, 3)
    xv = P[corner[..., 0], corner[..., 1], corner[..., 2]]           # (ne, 4, 3)
    ci = corner[..., 0] % nx
    cj = corner[..., 1] % ny
    tv = (corner[..., 2] * ny + cj) * nx + ci
    nv = nx * ny * (nz + 1)

    # region attribute by centroid
    regs = stack.regions()
    cen = xv.mean(axis=1)
    zc = cen[:, 2]
    attr = np.zeros(len(tv), dtype=np.int32)
    s = stack.slabs
    slab = np.clip(np.searchsorted(np.array(s[1:-1]), zc, side="right"), 0, len(s) - 2)
    for ridx, r in enumerate(regs, start=1):
        if r["kind"] == "background":
            attr[(slab == r["slab"]) & (zc >= stack.z_min) & (zc <= stack.z_max)] = ridx
    for ridx, r in enumerate(regs, start=1):
        if r["kind"] != "frustum":
            continue
        f = stack.frustums[r["frustum"]]
        d = f.inset(zc)
        inside = ((slab == r["slab"]) & (zc >= stack.z_min) & (zc <= stack.z_max)
                  & (zc >= f.z_lo) & (zc <= f.z_hi)
                  & (cen[:, 0] >= f.x0 + d) & (cen[:, 0] <= f.x1 - d)
                  & (cen[:, 1] >= f.y0 + d * (f.y0 > 0)) & (cen[:, 1] <= f.y1 - d * (f.y1 < stack.ly)))
        attr[inside] = ridx
    attr[zc < stack.z_min] = len(regs) - 1
    attr[zc > stack.z_max] = len(regs)
    if (attr == 0).any():  # pragma: no cover - geometry bug guard
        raise RuntimeError("unassigned elements")
    return TetMesh(tv=tv.astype(np.int64), xv=xv, attr=attr, nv=int(nv), grid=(nx, ny, nz))


def dofs_per_cube(p: int) -> int:
    """ND DOFs per Kuhn-subdivided periodic hex: 7 edges, 12 faces, 6 tets."""
    return 7 * p + 12 * p * (p - 1) + 6 * (p * (p - 1) * (p - 2) // 2)


def h_for_target_dofs(stack: Stack, p: int, ndof: float) -> float:
    vol = stack.lx * stack.ly * (stack.z_max - stack.z_min + 2 * stack.pml_thick)
    ncubes = ndof / dofs_per_cube(p)
    return (vol / ncubes) ** (1.0 / 3.0)
