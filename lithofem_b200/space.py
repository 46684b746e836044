"""ND finite element space on a ``TetMesh`` and the per-mesh assembly data.

Produces exactly the arrays the reference's GPU path consumes
(``AsmData``, solver/asm_data.inc:77-97), which the reference extracts from
MFEM in ``extract_asm_data`` (asm_data.inc:99-173):

* ``dof`` / ``sign``: decoded global DOF index and +-1 per element DOF
  (MFEM's negative-index encoding d < 0 -> -1 - d with sign -1,
  asm_data.inc:135-140);
* ``fo``: the 4 face orientations 0..5 per element (p >= 2);
* ``attr``, and the affine geometry ``J`` (row-major, J[i][j] = d x_i / d xi_j),
  ``Jinv``, ``detJ`` (> 0), ``v0`` (image of the reference origin);
* the two reference rules with their basis/curl tables (asm_data.inc:108-116).

DOF numbering follows the MFEM finite element space layout: all edge DOFs
(edge-major, p per edge, oriented from the lower to the higher global vertex
id), then face DOFs (p(p-1) per face), then element-interior DOFs.  A face's
global vertex order is the local order of the first element that references
it (that element sees orientation 0).  Orientation codes: the element-local
face vertex sequence (a, b, c) equals (G[pi(0)], G[pi(1)], G[pi(2)]) for the
global order G, with pi = FACE_PERMS[code]; local face DOF pairs then relate
to the global ones by the 2x2 matrix ``face_tinv(code)``, which is the block
the reference's dual transform applies (asm_data.inc:337-369).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import TetMesh
from .ndbasis import TET_EDGES, TET_FACES, face_points, nd_dofs, ref_tables
from .problem import Problem
from .quadrature import tet_rule

FACE_PERMS = ((0, 1, 2), (1, 0, 2), (1, 2, 0), (2, 1, 0), (2, 0, 1), (0, 2, 1))


def face_tinv(code: int) -> np.ndarray:
    """2x2 M with (local tangent pair) = M (global tangent pair) as functionals.

    Local tangents (b - a, c - a) expressed in the global ones (B - A, C - A)
    for the face permutation ``FACE_PERMS[code]``.
    """
    G = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])  # A, B, C in (T1, T2) coords
    pi = FACE_PERMS[code]
    a, b, c = G[pi[0]], G[pi[1]], G[pi[2]]
    return np.array([b - a, c - a])


def tinv_table() -> np.ndarray:
    """(24,) column-major 2x2 blocks per orientation, the layout of the
    reference's ``asm_nd_TInv`` (asm_data.inc:26-34)."""
    out = np.zeros(24)
    for o in range(6):
        M = face_tinv(o)
        out[4 * o:4 * o + 4] = [M[0, 0], M[1, 0], M[0, 1], M[1, 1]]
    return out


@dataclass
class AsmRefRule:
    nq: int
    ip: np.ndarray       # (nq*3,)
    w: np.ndarray        # (nq,)
    vshape: np.ndarray   # (nq*nd*3,)
    curl: np.ndarray     # (nq*nd*3,)


@dataclass
class AsmData:
    ne: int
    nd: int
    p: int
    height: int
    has_kpar: bool
    dof: np.ndarray       # int32 (ne*nd,)
    sign: np.ndarray      # f64 (ne*nd,)
    fo: np.ndarray        # int32 (ne*4,) or empty for p = 1
    attr: np.ndarray      # int32 (ne,)
    J: np.ndarray         # f64 (ne*9,)
    Jinv: np.ndarray      # f64 (ne*9,)
    detJ: np.ndarray      # f64 (ne,)
    v0: np.ndarray        # f64 (ne*3,)
    rule_cc: AsmRefRule
    rule_mass: AsmRefRule
    I: np.ndarray | None = None      # int32 (height+1,)
    Jcol: np.ndarray | None = None   # int32 (nnz,)
    ess: np.ndarray | None = None    # int32 sorted essential DOF list

    @property
    def nnz(self) -> int:
        return 0 if self.Jcol is None else int(self.Jcol.shape[0])


def _rule(p: int, degree: int) -> AsmRefRule:
    r = tet_rule(degree)
    v, c = ref_tables(p, r.ip)
    return AsmRefRule(nq=r.nq, ip=np.ascontiguousarray(r.ip.reshape(-1)),
                      w=r.w.copy(), vshape=v, curl=c)


def _first_occurrence_index(keys: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Global ids numbered by first appearance in row order of ``keys``.

    Returns (ids per row, row index of each id's first occurrence).
    """
    uniq, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    return rank[inv.reshape(-1)], first[order]


def build_asm_data(mesh: TetMesh, p: int, prob: Problem | None = None,
                   build_csr: bool = False, local_order_seed: int | None = None) -> AsmData:
    """Space + per-mesh data.

    Element-local vertex order: ascending global id, or (``local_order_seed``)
    a seeded random order, which exercises every edge sign and the face
    orientations {0, 1, 3, 5} of consistently oriented meshes; in both cases
    the last two vertices are swapped where needed so that detJ > 0
    (positively oriented, as extract_asm_data requires).
    """
    ne = mesh.ne
    nd = nd_dofs(p)
    if local_order_seed is None:
        order = np.argsort(mesh.tv, axis=1, kind="stable")
    else:
        rng = np.random.default_rng(local_order_seed)
        order = np.argsort(rng.random((ne, 4)), axis=1)
    tv = np.take_along_axis(mesh.tv, order, axis=1)
    xv = np.take_along_axis(mesh.xv, order[:, :, None], axis=1)
    Jm = np.stack([xv[:, 1] - xv[:, 0], xv[:, 2] - xv[:, 0], xv[:, 3] - xv[:, 0]], axis=2)
    det = np.linalg.det(Jm)
    neg = det < 0
    tv[neg] = tv[neg][:, [0, 1, 3, 2]]
    xv[neg] = xv[neg][:, [0, 1, 3, 2]]
    Jm = np.stack([xv[:, 1] - xv[:, 0], xv[:, 2] - xv[:, 0], xv[:, 3] - xv[:, 0]], axis=2)
    det = np.linalg.det(Jm)
    if (det <= 0).any():
        raise RuntimeError("degenerate element")
    Jinv = np.linalg.inv(Jm)

    # ---- edges ----
    le = np.array(TET_EDGES)
    ev = tv[:, le]                                  # (ne, 6, 2)
    ekey = np.sort(ev, axis=2).reshape(-1, 2)
    eid, _ = _first_occurrence_index(ekey)
    eid = eid.reshape(ne, 6)
    nE = int(eid.max()) + 1
    esgn = np.where(ev[:, :, 0] < ev[:, :, 1], 1, -1)

    # ---- faces ----
    lf = np.array(TET_FACES)
    fv = tv[:, lf]                                  # (ne, 4, 3)
    fkey = np.sort(fv, axis=2).reshape(-1, 3)
    fid, first = _first_occurrence_index(fkey)
    fid = fid.reshape(ne, 4)
    nF = int(fid.max()) + 1
    gorder = fv.reshape(-1, 3)[first]               # (nF, 3) global vertex order
    G = gorder[fid]                                 # (ne, 4, 3)
    pos = np.argmax(fv[:, :, :, None] == G[:, :, None, :], axis=3)  # (ne,4,3) pi
    code_of = {perm: c for c, perm in enumerate(FACE_PERMS)}
    pkey = pos[..., 0] * 9 + pos[..., 1] * 3 + pos[..., 2]
    lut = np.full(27, -1)
    for perm, c in code_of.items():
        lut[perm[0] * 9 + perm[1] * 3 + perm[2]] = c
    fo = lut[pkey]
    if (fo < 0).any():  # pragma: no cover
        raise RuntimeError("face orientation failed")
    # boundary faces: referenced by one element only (periodic sides paired)
    fcount = np.bincount(fid.reshape(-1), minlength=nF)

    # ---- DOF map ----
    ndof_e = p
    ndof_f = p * (p - 1)
    nint = nd - 6 * ndof_e - 4 * ndof_f
    n_edge_dofs = nE * ndof_e
    n_face_dofs = nF * ndof_f
    height = n_edge_dofs + n_face_dofs + ne * nint
    dof = np.zeros((ne, nd), dtype=np.int64)
    sign = np.ones((ne, nd))
    k = np.arange(p)
    for le_i in range(6):
        s = esgn[:, le_i:le_i + 1]
        kk = np.where(s > 0, k[None, :], p - 1 - k[None, :])
        dof[:, le_i * p:(le_i + 1) * p] = eid[:, le_i:le_i + 1] * p + kk
        sign[:, le_i * p:(le_i + 1) * p] = s
    if p >= 2:
        fp = face_points(p)
        npt = len(fp)
        sig = np.zeros((6, npt), dtype=np.int64)
        for code, pi in enumerate(FACE_PERMS):
            for i, lam in enumerate(fp):
                mu = np.zeros(3)
                for t in range(3):
                    mu[pi[t]] = lam[t]
                j = int(np.argmin(np.abs(fp - mu[None, :]).sum(axis=1)))
                if np.abs(fp[j] - mu).max() > 1e-12:  # pragma: no cover
                    raise RuntimeError("face points not orientation-invariant")
                sig[code, i] = j
        base = 6 * p
        for f in range(4):
            s = sig[fo[:, f]]                        # (ne, npt)
            for i in range(npt):
                for t in range(2):
                    col = base + f * ndof_f + 2 * i + t
                    dof[:, col] = n_edge_dofs + fid[:, f] * ndof_f + 2 * s[:, i] + t
    if nint:
        off = n_edge_dofs + n_face_dofs
        dof[:, nd - nint:] = off + np.arange(ne)[:, None] * nint + np.arange(nint)[None, :]

    # essential DOFs: every boundary face (after periodic pairing only the
    # z caps remain) with its edges
    bf = fcount == 1
    ess = []
    el_b, lf_b = np.nonzero(bf[fid])
    if len(el_b):
        fedges = {0: (3, 4, 5), 1: (2, 5, 1), 2: (0, 4, 2), 3: (1, 3, 0)}
        for f in range(4):
            m = lf_b == f
            els = el_b[m]
            for le_i in fedges[f]:
                ess.append(dof[els, le_i * p:(le_i + 1) * p].reshape(-1))
            if p >= 2:
                ess.append(dof[els, 6 * p + f * ndof_f:6 * p + (f + 1) * ndof_f].reshape(-1))
    ess_arr = np.unique(np.concatenate(ess)).astype(np.int32) if ess else np.zeros(0, np.int32)

    ad = AsmData(
        ne=ne, nd=nd, p=p, height=int(height),
        has_kpar=bool(prob.has_kpar) if prob is not None else False,
        dof=np.ascontiguousarray(dof.reshape(-1).astype(np.int32)),
        sign=np.ascontiguousarray(sign.reshape(-1)),
        fo=np.ascontiguousarray(fo.reshape(-1).astype(np.int32)) if p >= 2
        else np.zeros(0, np.int32),
        attr=np.ascontiguousarray(mesh.attr.astype(np.int32)),
        J=np.ascontiguousarray(Jm.reshape(-1)),
        Jinv=np.ascontiguousarray(Jinv.reshape(-1)),
        detJ=np.ascontiguousarray(det),
        v0=np.ascontiguousarray(xv[:, 0].reshape(-1)),
        rule_cc=_rule(p, max(0, 2 * p - 2)),
        rule_mass=_rule(p, 2 * p),
        ess=ess_arr,
    )
    if build_csr:
        ad.I, ad.Jcol = csr_symbolic(ad)
    return ad


def build_asm_data_device(mesh: TetMesh, p: int, prob: Problem | None = None, gpu_id: int = 0,
                          build_csr: bool = False) -> AsmData:
    """build_asm_data (ascending local vertex order) with the extraction on
    the device (lfasm_extract): local order, Jacobians, edge and face
    numbering by first occurrence, face orientations, the DOF map and the
    essential DOFs.  The integer arrays equal build_asm_data's; J and v0
    too; Jinv and detJ come from the adjugate and agree to rounding."""
    import ctypes as ct

    from . import _lib
    from ._abi import c_double_p, c_int_p
    ne = mesh.ne
    nd = nd_dofs(p)
    tv = np.ascontiguousarray(mesh.tv, dtype=np.int32)
    xv = np.ascontiguousarray(mesh.xv, dtype=np.float64)
    dof = np.empty(ne * nd, dtype=np.int32)
    sign = np.empty(ne * nd)
    fo = np.empty(ne * 4 if p >= 2 else 0, dtype=np.int32)
    J = np.empty(ne * 9)
    Jinv = np.empty(ne * 9)
    det = np.empty(ne)
    v0 = np.empty(ne * 3)
    cap = ne * nd
    ess = np.empty(cap, dtype=np.int32)
    height, n_ess = ct.c_int(), ct.c_int()
    ip, dp = (lambda a: a.ctypes.data_as(c_int_p)), (lambda a: a.ctypes.data_as(c_double_p))
    rc = _lib.lib().lfasm_extract(int(gpu_id), ne, int(mesh.nv), int(p), ip(tv), dp(xv), ip(dof),
                                  dp(sign), ip(fo) if p >= 2 else None, dp(J), dp(Jinv), dp(det),
                                  dp(v0), ip(ess), cap, ct.byref(height), ct.byref(n_ess))
    _lib.check(rc)
    ad = AsmData(
        ne=ne, nd=nd, p=p, height=int(height.value),
        has_kpar=bool(prob.has_kpar) if prob is not None else False,
        dof=dof, sign=sign, fo=fo, attr=np.ascontiguousarray(mesh.attr.astype(np.int32)),
        J=J, Jinv=Jinv, detJ=det, v0=v0,
        rule_cc=_rule(p, max(0, 2 * p - 2)), rule_mass=_rule(p, 2 * p),
        ess=ess[:n_ess.value].copy(),
    )
    if build_csr:
        ad.I, ad.Jcol = csr_symbolic(ad)
    return ad


def csr_symbolic(ad: AsmData) -> tuple[np.ndarray, np.ndarray]:
    """Per-row sorted unique columns of the element DOF graph.

    Host restatement of ``build_csr_symbolic`` (asm_data.inc:178-210), used for
    small meshes and as a cross-check of the device builder.
    """
    nd = ad.nd
    d = ad.dof.reshape(ad.ne, nd).astype(np.int64)
    rows = np.repeat(d, nd, axis=1).reshape(-1)
    cols = np.tile(d, (1, nd)).reshape(-1)
    key = np.unique(rows * ad.height + cols)
    r = key // ad.height
    c = key % ad.height
    I = np.zeros(ad.height + 1, dtype=np.int64)
    np.add.at(I, r + 1, 1)
    I = np.cumsum(I)
    return I.astype(np.int32), c.astype(np.int32)
