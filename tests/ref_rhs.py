"""Test infrastructure: a right-hand side integrated from given point sources.

``rhs_from_points`` forms b = sum_e sum_q w_q detJ_e sign . T_e^T (v_k(x_q) .
f_eq) for point source values f (ne, nq, 3) at the mass-rule points: the
physical vector shapes v = vshape . Jinv, the dual face transform applied to
the element vector's face pairs (TInv(fo) rows, solver/asm_data.inc:337-369),
DOF signs, and essential rows zeroed (form_rhs_only,
solver/lithofem_solve.cpp:732-742).  Fed with the reference's own
ScatterSource values it gives the reference's source integrated with this
repository's quadrature, independent of the oracle's code.
"""

from __future__ import annotations

import numpy as np

from lithofem_b200 import space


def rhs_from_points(ad, f: np.ndarray, ess=None, eliminate: bool = True) -> np.ndarray:
    rm = ad.rule_mass
    nd, ne = ad.nd, ad.ne
    vs = np.asarray(rm.vshape).reshape(rm.nq, nd, 3)
    Ji = ad.Jinv.reshape(ne, 3, 3)
    pv = np.einsum("qkj,ejd->eqkd", vs, Ji)                 # physical shapes
    w = np.asarray(rm.w)[None, :] * ad.detJ[:, None]        # (ne, nq)
    be = np.einsum("eq,eqkd,eqd->ek", w, pv, f)
    if ad.p >= 2:
        tinv = space.tinv_table().reshape(6, 4)
        fo = ad.fo.reshape(ne, 4)
        foff, ntd = 6 * ad.p, ad.p * (ad.p - 1)
        for fc in range(4):
            T = tinv[fo[:, fc]]                             # (ne, 4)
            for i in range(ntd // 2):
                d0 = foff + fc * ntd + 2 * i
                a, b = be[:, d0].copy(), be[:, d0 + 1].copy()
                be[:, d0] = T[:, 0] * a + T[:, 1] * b
                be[:, d0 + 1] = T[:, 2] * a + T[:, 3] * b
    out = np.zeros(ad.height, dtype=np.complex128)
    np.add.at(out, ad.dof.reshape(ne, nd), ad.sign.reshape(ne, nd) * be)
    if eliminate and ess is not None and len(ess):
        out[np.asarray(ess)] = 0.0
    return out
