"""Polygon-hole meshes of the batched workload: geometry, walls, periodicity,
H(curl) conformity and the seeded batch parameters."""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs, ndbasis
from tests.test_basis import _tangential_jump


def _vertices(ad):
    ne = ad.ne
    J = ad.J.reshape(ne, 3, 3)
    v0 = ad.v0.reshape(ne, 3)
    return np.stack([v0, v0 + J[:, :, 0], v0 + J[:, :, 1], v0 + J[:, :, 2]], axis=1)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_volumes(p):
    """Cell volume, and the hole volume equals the integral of the mitre-offset
    section area (quadratic in the offset, so Simpson is exact)."""
    c = configs.small_poly_case(p, 6.0, seed=11 + p)
    st, hole, ad = c.stack, c.stack.frustums[0], c.ad
    vol = st.lx * st.ly * (st.z_max - st.z_min + 2 * st.pml_thick)
    assert abs(ad.detJ.sum() / 6.0 - vol) / vol < 1e-12
    regs = st.regions()
    hole_attr = [i + 1 for i, r in enumerate(regs) if r["kind"] == "frustum"]
    assert len(hole_attr) == 1
    v_hole = ad.detJ[ad.attr == hole_attr[0]].sum() / 6.0
    z = np.linspace(hole.z_lo, hole.z_hi, 3)
    a = [hole.area(float(hole.inset(zz))) for zz in z]
    exact = (hole.z_hi - hole.z_lo) / 6.0 * (a[0] + 4 * a[1] + a[2])
    assert abs(v_hole - exact) / exact < 1e-10


def test_walls_lie_on_the_mitre_planes():
    """Every face between the hole and the absorber lies on one wall plane:
    inward distance to a base edge line = |z - z0| / tan(alpha)."""
    c = configs.small_poly_case(2, 6.0, seed=21)
    st, hole, ad = c.stack, c.stack.frustums[0], c.ad
    regs = st.regions()
    ah = [i + 1 for i, r in enumerate(regs) if r["kind"] == "frustum"][0]
    ab = [i + 1 for i, r in enumerate(regs) if r["kind"] == "background" and r["slab"] == 0][0]
    xv = _vertices(ad)
    faces = {}
    for e in np.nonzero((ad.attr == ah) | (ad.attr == ab))[0]:
        for tri in ndbasis.TET_FACES:
            k = tuple(sorted(map(tuple, np.round(xv[e, list(tri)], 9))))
            faces.setdefault(k, []).append(ad.attr[e])
    V = np.asarray(hole.verts)
    E = np.roll(V, -1, axis=0) - V
    N = np.stack([-E[:, 1], E[:, 0]], axis=1) / np.linalg.norm(E, axis=1)[:, None]
    walls = 0
    for k, at in faces.items():
        if sorted(at) != sorted([ah, ab]):
            continue
        P = np.array(k)
        d_in = np.einsum("pvk,vk->pv", P[:, None, :2] - V[None, :, :], N)
        want = hole.inset(P[:, 2])
        ok = np.abs(d_in - want[:, None]).max(axis=0) < 1e-9
        assert ok.any(), k
        walls += 1
    assert walls > 20


def test_periodic_identification():
    """Vertices sharing a topological id differ by lattice vectors only."""
    c = configs.small_poly_case(1, 0.0, seed=5, local_order_seed=None)
    from lithofem_b200.mesh_poly import build_poly_mesh
    m = build_poly_mesh(c.stack, c.stack.frustums[0], 2.0)
    lx, ly = c.stack.lx, c.stack.ly
    ref = {}
    n_wrapped = 0
    for t, x in zip(m.tv.ravel(), m.xv.reshape(-1, 3)):
        if t in ref:
            d = x - ref[t]
            assert abs(d[2]) < 1e-12
            assert abs(d[0] / lx - round(d[0] / lx)) < 1e-12
            assert abs(d[1] / ly - round(d[1] / ly)) < 1e-12
            n_wrapped += int(abs(d[0]) > 1e-9 or abs(d[1]) > 1e-9)
        else:
            ref[t] = x
    assert n_wrapped > 0


@pytest.mark.parametrize("p", [1, 2, 3])
def test_hcurl_conformity(p):
    c = configs.small_poly_case(p, 6.0, seed=31 + p, h={1: 2.4, 2: 3.2, 3: 4.4}[p])
    worst, cnt = _tangential_jump(c)
    assert cnt > 50
    assert worst < 1e-11, worst


def test_batch_parameters():
    cases = configs.batch_config(scale=0.01, n=4)
    assert [c.p for c in cases] == [1, 2, 3, 1]
    for c in cases:
        hole = c.stack.frustums[0]
        assert 3 <= len(hole.verts) <= 8
        assert 80.0 <= hole.alpha <= 90.0
        assert 40.0 <= hole.h <= 70.0
        assert (c.ad.detJ > 0).all()
    assert len({c.stack.frustums[0].verts for c in cases}) == 4
