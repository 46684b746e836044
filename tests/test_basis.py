"""Reference element, quadrature and ND space (CPU).

Mirrors the reference's table/geometry unit checks (U1/U2,
solver/asm_test.cpp:49-125) for this repository's own basis and mesher,
plus the H(curl) conformity that the reference inherits from MFEM.
"""

from __future__ import annotations

from math import factorial

import numpy as np
import pytest

from lithofem_b200 import configs, mesh as M, ndbasis, quadrature, space

# the reference's face-DOF 2x2 tables (solver/asm_data.inc:26-34), golden values
REF_TINV = np.array([1, 0, 0, 1, -1, -1, 0, 1, -1, -1, 1, 0,
                     1, 0, -1, -1, 0, 1, -1, -1, 0, 1, 1, 0], dtype=float)
REF_T = np.array([1, 0, 0, 1, -1, -1, 0, 1, 0, 1, -1, -1,
                  1, 0, -1, -1, -1, -1, 1, 0, 0, 1, 1, 0], dtype=float)


@pytest.mark.parametrize("deg", [0, 2, 4, 6])
def test_rule_exactness(deg):
    r = quadrature.tet_rule(deg)
    assert abs(r.w.sum() - 1.0 / 6.0) < 1e-15
    for a in range(deg + 1):
        for b in range(deg + 1 - a):
            for c in range(deg + 1 - a - b):
                ex = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
                got = (r.w * r.ip[:, 0] ** a * r.ip[:, 1] ** b * r.ip[:, 2] ** c).sum()
                assert abs(got - ex) < 2e-16, (deg, a, b, c)
    assert r.nq == {0: 1, 2: 4, 4: 11, 6: 24}[deg]


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_nd_duality_and_size(p):
    el = ndbasis.nd_element(p)
    assert el.nd == p * (p + 2) * (p + 3) // 2
    V = np.einsum("ikd,id->ik", el.vshape(el.dof_pts), el.dof_tan)
    assert np.abs(V - np.eye(el.nd)).max() < 1e-12


def test_whitney_p1():
    el = ndbasis.nd_element(1)
    x = np.array([[0.1, 0.2, 0.3]])
    lam = np.array([1 - x.sum(), *x[0]])
    grads = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    for k, (a, b) in enumerate(ndbasis.TET_EDGES):
        w = lam[a] * grads[b] - lam[b] * grads[a]
        assert np.allclose(el.vshape(x)[0, k], w, atol=1e-14)
        assert np.allclose(el.curl(x)[0, k], 2 * np.cross(grads[a], grads[b]), atol=1e-13)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_curl_matches_finite_difference(p):
    el = ndbasis.nd_element(p)
    x = np.array([0.21, 0.17, 0.33])
    h = 1e-6

    def u(y):
        return el.vshape(y[None])[0]

    J = np.zeros((el.nd, 3, 3))
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        J[:, :, j] = (u(x + e) - u(x - e)) / (2 * h)
    curl = np.stack([J[:, 2, 1] - J[:, 1, 2], J[:, 0, 2] - J[:, 2, 0], J[:, 1, 0] - J[:, 0, 1]], 1)
    assert np.abs(curl - el.curl(x[None])[0]).max() < 1e-6


def test_face_tables_equal_reference():
    assert np.array_equal(space.tinv_table(), REF_TINV)
    # T is the inverse of TInv blockwise
    for o in range(6):
        Ti = REF_TINV[4 * o:4 * o + 4].reshape(2, 2, order="F")
        T = REF_T[4 * o:4 * o + 4].reshape(2, 2, order="F")
        assert np.allclose(Ti @ T, np.eye(2))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_geometry_and_volume(p):
    c = configs.small_case("hole", p, 0.0)
    ad = c.ad
    J = ad.J.reshape(-1, 3, 3)
    assert (ad.detJ > 0).all()
    assert np.allclose(np.linalg.det(J), ad.detJ, rtol=1e-13)
    assert np.allclose(np.einsum("eij,ejk->eik", J, ad.Jinv.reshape(-1, 3, 3)), np.eye(3), atol=1e-12)
    st = c.stack
    vol = st.lx * st.ly * (st.z_max - st.z_min + 2 * st.pml_thick)
    assert abs(ad.detJ.sum() / 6.0 - vol) / vol < 1e-12


def _tangential_jump(case, n_faces=400):
    ad = case.ad
    p, nd, ne = ad.p, ad.nd, ad.ne
    el = ndbasis.nd_element(p)
    rng = np.random.default_rng(0)
    u = rng.standard_normal(ad.height)
    dof = ad.dof.reshape(ne, nd)
    sg = ad.sign.reshape(ne, nd)
    fo = ad.fo.reshape(ne, 4) if p >= 2 else None
    Jm = ad.J.reshape(ne, 3, 3)
    Ji = ad.Jinv.reshape(ne, 3, 3)
    v0 = ad.v0.reshape(ne, 3)

    def coef(e):
        g = sg[e] * u[dof[e]]
        c = g.copy()
        if p >= 2:
            for f in range(4):
                Mt = space.face_tinv(fo[e, f])
                for i in range(p * (p - 1) // 2):
                    d0 = 6 * p + f * p * (p - 1) + 2 * i
                    c[d0:d0 + 2] = Mt @ g[d0:d0 + 2]
        return c

    def field(e, X):
        xi = np.linalg.solve(Jm[e], (X - v0[e]).T).T
        return np.einsum("k,qkd->qd", coef(e), el.vshape(xi)) @ Ji[e]

    xv = np.stack([v0, v0 + Jm[:, :, 0], v0 + Jm[:, :, 1], v0 + Jm[:, :, 2]], axis=1)
    keys = {}
    for e in range(ne):
        for f, tri in enumerate(ndbasis.TET_FACES):
            k = tuple(sorted(map(tuple, np.round(xv[e, list(tri)], 9))))
            keys.setdefault(k, []).append((e, tri))
    worst, cnt = 0.0, 0
    for k, lst in keys.items():
        if len(lst) != 2:
            continue
        (e1, t1), (e2, _) = lst
        pts = xv[e1, list(t1)]
        X = rng.dirichlet([1, 1, 1], size=3) @ pts
        nrm = np.cross(pts[1] - pts[0], pts[2] - pts[0])
        nrm /= np.linalg.norm(nrm)
        a, b = field(e1, X), field(e2, X)
        ta = a - np.outer(a @ nrm, nrm)
        tb = b - np.outer(b @ nrm, nrm)
        worst = max(worst, np.abs(ta - tb).max() / max(np.abs(ta).max(), 1e-300))
        cnt += 1
        if cnt >= n_faces:
            break
    return worst, cnt


@pytest.mark.parametrize("p", [1, 2, 3])
def test_hcurl_conformity(p):
    """Tangential traces of a random global field agree across interior faces."""
    c = configs.small_case("hole", p, 6.0, seed=3, h={1: 2.4, 2: 3.0, 3: 4.0}[p])
    worst, cnt = _tangential_jump(c)
    assert cnt > 50
    assert worst < 1e-11, worst


def test_face_orientation_coverage():
    """Seeded local orders give fo in {0,1,3,5} (mask 43), as the reference
    asserts for consistently oriented meshes (tests/test_asm_v25.py:126-140)."""
    c = configs.small_case("hole", 2, 0.0, seed=5)
    seen = 0
    for o in np.unique(c.ad.fo):
        seen |= 1 << int(o)
    assert seen == 43


def test_region_attributes_and_pml():
    st = configs.contact_hole_stack()
    regs = st.regions()
    kinds = [r["kind"] for r in regs]
    assert kinds == ["background", "frustum", "background", "pml_bottom", "pml_top"]
    assert regs[3]["eps"] == configs.ABSORBER and regs[4]["eps"] == 1.0
    c = configs.small_case("hole", 1, 0.0)
    counts = np.bincount(c.ad.attr)
    assert (counts[1:] > 0).all()


def test_essential_dofs_are_z_caps():
    c = configs.small_case("slab", 2, 0.0)
    ad = c.ad
    zlo = c.stack.z_min - c.stack.pml_thick
    zhi = c.stack.z_max + c.stack.pml_thick
    # every essential dof belongs to an element touching a cap
    ne, nd = ad.ne, ad.nd
    J = ad.J.reshape(ne, 3, 3)
    v0 = ad.v0.reshape(ne, 3)
    zs = np.stack([v0[:, 2], v0[:, 2] + J[:, 2, 0], v0[:, 2] + J[:, 2, 1], v0[:, 2] + J[:, 2, 2]], 1)
    touch = (np.isclose(zs, zlo).sum(1) >= 3) | (np.isclose(zs, zhi).sum(1) >= 3)
    cap_dofs = np.unique(ad.dof.reshape(ne, nd)[touch])
    assert np.isin(ad.ess, cap_dofs).all()
    assert len(ad.ess) > 0
