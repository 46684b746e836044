"""Structure of the assembled system on the GPU: complex symmetry at
k_par = 0 (the reference's MMS check, tests/test_mms.py:52-69), the Bloch
transpose relation A(k)^T = A(-k), and tiny meshes (one tet, one cube)
against the oracle."""

from __future__ import annotations

import copy

import numpy as np
import pytest
import scipy.sparse as sp

from lithofem_b200 import configs, mesh, problem, space
from lithofem_b200.asm import CROSS0, CROSS1, CURLCURL, KLK, MASS, AsmGpu, AsmGpuGlobal
from oracle import oracle

pytestmark = pytest.mark.gpu


def _matrix(c, prob, eliminate):
    g = AsmGpuGlobal(prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess) and g.Assemble(eliminate)
    I, J = g.DownloadCsr()
    v = g.DownloadValues()
    n = c.ad.height
    return sp.csr_matrix((v, J, I), shape=(n, n))


@pytest.mark.parametrize("kind,p", [("hole", 2), ("grating", 3), ("slab", 1)])
def test_complex_symmetric_at_zero_kpar(kind, p):
    c = configs.small_case(kind, p, 0.0, seed=13, h={1: 1.8, 2: 2.4, 3: 3.2}[p])
    assert not c.prob.has_kpar
    for elim in (False, True):
        A = _matrix(c, c.prob, elim)
        d = abs(A - A.T).max() / abs(A).max()
        assert d < 1e-12, (elim, d)


@pytest.mark.parametrize("kind,p", [("hole", 2), ("grating", 3)])
def test_bloch_transpose(kind, p):
    """A(kx, ky)^T = A(-kx, -ky): the cross terms swap and K -> -K."""
    c = configs.small_case(kind, p, 6.0, seed=13, h={2: 2.4, 3: 3.2}[p])
    assert c.prob.has_kpar
    pm = copy.copy(c.prob)
    pm.kx, pm.ky = -c.prob.kx, -c.prob.ky
    A = _matrix(c, c.prob, False)
    B = _matrix(c, pm, False)
    d = abs(A.T - B).max() / abs(A).max()
    assert d < 1e-12, d
    assert abs(A - A.T).max() / abs(A).max() > 1e-6   # not symmetric itself


def _tiny(p, z_lo, cube):
    st = mesh.Stack(lx=4.0, ly=4.0, z_min=0.0, z_max=8.0, wavelength=configs.WAVELENGTH,
                    layers=[(0.0, 4.0, configs.ABSORBER)], pml_thickness_wavelengths=0.2)
    pr = problem.Problem.from_stack(st, p, configs.kpar_of(6.0))
    x0 = np.array([0.7, 0.9, z_lo])
    if cube:
        corners = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], float)
        tets = [[0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7], [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]]
        xv = np.array([[x0 + 1.3 * corners[v] for v in t] for t in tets])
        tv = np.array(tets, dtype=np.int64)
        nv = 8
    else:
        xv = np.array([[x0, x0 + [1.1, 0.1, 0.0], x0 + [0.2, 1.3, 0.1], x0 + [0.3, 0.2, 0.9]]])
        tv = np.array([[0, 1, 2, 3]], dtype=np.int64)
        nv = 4
    zc = xv[:, :, 2].mean(1)
    regs = st.regions()
    attr = np.where(zc < st.z_min, len(regs) - 1, 1).astype(np.int32)
    m = mesh.TetMesh(tv=tv, xv=xv, attr=attr, nv=nv)
    ad = space.build_asm_data(m, p, pr, build_csr=True, local_order_seed=11)
    return ad, pr


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("where", ["bulk", "pml"])
@pytest.mark.parametrize("cube", [False, True], ids=["1tet", "cube"])
def test_tiny_meshes(p, where, cube):
    z_lo = 1.0 if where == "bulk" else -2.5
    ad, pr = _tiny(p, z_lo, cube)
    g = AsmGpu(pr)
    assert g.Init(ad, 0)
    nb, npml = g.PathCounts()
    assert (npml if where == "pml" else nb) == ad.ne
    mm = MASS | CROSS0 | CROSS1 | KLK
    for mcc, mmass, te in [(CURLCURL, mm, True), (0, CROSS0, False), (CURLCURL, 0, False)]:
        assert g.ComputeLocal(mcc, mmass, te)
        ref = oracle.local(ad, pr, mcc, mmass, te)
        got = g.DownloadLocal()
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    gg = AsmGpuGlobal(pr)
    assert gg.Init(ad, 0) and gg.BuildGlobal(ad.ess)
    I, J = oracle.csr(ad)
    for elim in (False, True):   # all but the interior dofs of one tet are essential
        assert gg.Assemble(elim)
        ref = oracle.assemble(ad, pr, I, J, ad.ess, elim)
        assert np.abs(gg.DownloadValues() - ref).max() <= 1e-13 * np.abs(ref).max()
