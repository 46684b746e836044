"""Nedelec (first kind) H(curl) basis of order p on the reference tetrahedron.

The element of order p spans N_p = (P_{p-1})^3 + {q in (homogeneous P_p)^3 :
q . x = 0}, dimension nd = p (p + 2) (p + 3) / 2 (6 / 20 / 45 for p = 1 / 2 / 3,
the count the reference uses at solver/asm_data.inc:79-80).

The basis is the nodal (dual) basis of "tangential component at a point"
functionals, laid out in the element-local order of MFEM's
ND_TetrahedronElement, which the reference consumes through
``CalcVShape``/``CalcCurlShape`` (solver/asm_data.inc:47-73):

* 6 edges in the order (0,1), (0,2), (0,3), (1,2), (1,3), (2,3), p points
  each at the Gauss-Legendre abscissae of [0, 1], ordered from the first
  vertex to the second; tangent = edge vector (second minus first vertex);
* 4 faces in the order (1,2,3), (0,3,2), (0,1,3), (0,2,1); for a face
  (a, b, c) the p(p-1)/2 points are, for j = 0..p-2 and i = 0..p-2-j, the
  barycentric point (g[p-2-i-j], g[i], g[j]) / sum on (a, b, c), g the
  Gauss-Legendre abscissae of order p-1; each point carries the pair of
  tangents (b - a, c - a).  Face DOF d0 = 6p + f p(p-1) + 2i is the first
  of the pair (the layout the face-orientation transform of
  solver/asm_data.inc:337-369 addresses);
* interior: for k, j, i with i + j + k <= p-3, the point
  (g[i], g[j], g[k]) / (g[i] + g[j] + g[k] + g[p-3-i-j-k]) with the three
  unit axis tangents.

Polynomials are represented by coefficient arrays over the monomials
x^a y^b z^c with a + b + c <= p; curls are taken exactly on the
coefficients.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

import numpy as np

REF_VERTS = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0],
                      [0.0, 0.0, 1.0]])
TET_EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
TET_FACES = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))


def nd_dofs(p: int) -> int:
    return p * (p + 2) * (p + 3) // 2


def gl01(n: int) -> np.ndarray:
    """Gauss-Legendre abscissae on [0, 1], ascending."""
    x, _ = np.polynomial.legendre.leggauss(n)
    return np.sort(0.5 * (x + 1.0))


def face_points(p: int) -> np.ndarray:
    """Barycentric (on the face's own vertices (a, b, c)) face DOF points."""
    if p < 2:
        return np.zeros((0, 3))
    pm2 = p - 2
    g = gl01(p - 1)
    pts = []
    for j in range(pm2 + 1):
        for i in range(pm2 + 1 - j):
            w = g[i] + g[j] + g[pm2 - i - j]
            pts.append((g[pm2 - i - j] / w, g[i] / w, g[j] / w))
    return np.array(pts)


def _monomials(p: int) -> list[tuple[int, int, int]]:
    out = []
    for d in range(p + 1):
        for a in range(d, -1, -1):
            for b in range(d - a, -1, -1):
                out.append((a, b, d - a - b))
    return out


def _eval_monos(monos, x: np.ndarray) -> np.ndarray:
    """(npts, nmono) monomial values."""
    x = np.atleast_2d(x)
    out = np.empty((x.shape[0], len(monos)))
    for m, (a, b, c) in enumerate(monos):
        out[:, m] = x[:, 0] ** a * x[:, 1] ** b * x[:, 2] ** c
    return out


@dataclass(frozen=True)
class NDElement:
    """Nodal ND_p basis: ``coef`` (nd, 3, nmono) monomial coefficients."""

    p: int
    monos: tuple
    coef: np.ndarray
    dof_pts: np.ndarray   # (nd, 3)
    dof_tan: np.ndarray   # (nd, 3)

    @property
    def nd(self) -> int:
        return self.coef.shape[0]

    def vshape(self, x: np.ndarray) -> np.ndarray:
        """(npts, nd, 3) basis values at reference points."""
        mv = _eval_monos(self.monos, x)
        return np.einsum("qm,kdm->qkd", mv, self.coef)

    def curl(self, x: np.ndarray) -> np.ndarray:
        """(npts, nd, 3) basis curls at reference points."""
        return np.einsum("qm,kdm->qkd", _eval_monos(self.monos, x), self._curl_coef)

    @property
    def _curl_coef(self) -> np.ndarray:
        return _curl_coefficients(self.p, self.coef, self.monos)


def _deriv_matrix(monos, axis: int) -> np.ndarray:
    """D (nmono, nmono): coefficients of d/d(axis) of each monomial."""
    idx = {m: i for i, m in enumerate(monos)}
    D = np.zeros((len(monos), len(monos)))
    for i, m in enumerate(monos):
        if m[axis] == 0:
            continue
        mm = list(m)
        mm[axis] -= 1
        D[idx[tuple(mm)], i] = m[axis]
    return D


def _curl_coefficients(p, coef, monos) -> np.ndarray:
    Dx, Dy, Dz = (_deriv_matrix(monos, a) for a in range(3))
    ux, uy, uz = coef[:, 0, :], coef[:, 1, :], coef[:, 2, :]
    cx = uz @ Dy.T - uy @ Dz.T
    cy = ux @ Dz.T - uz @ Dx.T
    cz = uy @ Dx.T - ux @ Dy.T
    return np.stack([cx, cy, cz], axis=1)


def dof_layout(p: int) -> tuple[np.ndarray, np.ndarray]:
    """Element-local DOF points and tangents (reference coordinates)."""
    V = REF_VERTS
    pts, tans = [], []
    ge = gl01(p)
    for a, b in TET_EDGES:
        for s in ge:
            pts.append(V[a] + s * (V[b] - V[a]))
            tans.append(V[b] - V[a])
    fp = face_points(p)
    for a, b, c in TET_FACES:
        for lam in fp:
            x = lam[0] * V[a] + lam[1] * V[b] + lam[2] * V[c]
            pts.append(x)
            tans.append(V[b] - V[a])
            pts.append(x)
            tans.append(V[c] - V[a])
    if p >= 3:
        pm3 = p - 3
        g = gl01(p - 2)
        for k in range(pm3 + 1):
            for j in range(pm3 + 1 - k):
                for i in range(pm3 + 1 - j - k):
                    w = g[i] + g[j] + g[k] + g[pm3 - i - j - k]
                    x = np.array([g[i], g[j], g[k]]) / w
                    for t in np.eye(3):
                        pts.append(x)
                        tans.append(t)
    return np.array(pts), np.array(tans)


@lru_cache(maxsize=None)
def nd_element(p: int) -> NDElement:
    if p < 1:
        raise ValueError("ND order must be >= 1")
    monos = _monomials(p)
    nm = len(monos)
    gen = []
    for m, e in enumerate(monos):
        if sum(e) <= p - 1:
            for d in range(3):
                c = np.zeros((3, nm))
                c[d, m] = 1.0
                gen.append(c)
    idx = {m: i for i, m in enumerate(monos)}
    for e in monos:
        if sum(e) != p - 1:
            continue
        for d in range(3):
            # x cross (e_d * mono): e_x -> (0, z, -y); e_y -> (-z, 0, x); e_z -> (y, -x, 0)
            c = np.zeros((3, nm))

            def add(comp, var, sgn):
                ee = list(e)
                ee[var] += 1
                c[comp, idx[tuple(ee)]] += sgn

            if d == 0:
                add(1, 2, 1.0)
                add(2, 1, -1.0)
            elif d == 1:
                add(0, 2, -1.0)
                add(2, 0, 1.0)
            else:
                add(0, 1, 1.0)
                add(1, 0, -1.0)
            gen.append(c)
    G = np.array([g.reshape(-1) for g in gen])
    _, s, vt = np.linalg.svd(G, full_matrices=False)
    nd = nd_dofs(p)
    rank = int((s > 1e-10 * s[0]).sum())
    if rank != nd:  # pragma: no cover - algebraic identity
        raise RuntimeError(f"ND_{p} space rank {rank} != {nd}")
    span = vt[:nd].reshape(nd, 3, nm)
    pts, tans = dof_layout(p)
    mv = _eval_monos(monos, pts)                     # (nd, nm)
    vals = np.einsum("im,jdm->ijd", mv, span)        # (dof i, span j, 3)
    Vdm = np.einsum("ijd,id->ij", vals, tans)        # DOF_i(span_j)
    coef = np.einsum("jk,jdm->kdm", np.linalg.inv(Vdm), span)
    return NDElement(p=p, monos=tuple(monos), coef=coef, dof_pts=pts, dof_tan=tans)


def ref_tables(p: int, ip: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(vshape, curl) tables at points ``ip``, each flat [q*nd*3 + k*3 + d].

    Same layout as the reference's AsmRefRule (solver/asm_data.inc:38-45).
    """
    el = nd_element(p)
    return (np.ascontiguousarray(el.vshape(ip).reshape(-1)),
            np.ascontiguousarray(el.curl(ip).reshape(-1)))
