"""The benchmark's full-size system (line grating, p = 3, theta = 6 deg,
1,346,625 DOF, 115,149,195 nnz), checked through properties that do not
depend on size, where the oracle would need minutes for the whole mesh:

* CSR structure: row pointer monotone, columns strictly increasing in every
  row, every row holding its diagonal; values bitwise equal run to run.
* The Bloch transpose A(k)^T = A(-k) over every entry (a device sort).
* Linearity in the per-element permittivity:
  A(eps1) + A(eps2) = 2 A((eps1 + eps2) / 2).
* lfasm_spmv against an independent product on the same device CSR.
* Oracle parity on a seeded sample of the mesh's elements, bulk and PML
  alike: the full mesh's geometry, orientations and signs, assembled alone.
"""

from __future__ import annotations

import copy
import dataclasses

import numpy as np
import pytest

from lithofem_b200 import configs, space
from lithofem_b200.asm import AsmGpuGlobal
from oracle import oracle

pytestmark = pytest.mark.gpu

NNZ_C3 = 115_149_195


@pytest.fixture(scope="module")
def c3():
    return configs.config(3)


def _assemble(prob, ad, eliminate=True):
    g = AsmGpuGlobal(prob)
    assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(eliminate)
    return g


def _views(g):
    import torch
    I, J, V = (torch.as_tensor(x, device="cuda") for x in g.DeviceCsrViews())
    return I, J, V


def _rows(I):
    import torch
    n = I.numel() - 1
    return torch.repeat_interleave(torch.arange(n, device=I.device), (I[1:] - I[:-1]).long())


def test_structure_and_determinism(c3):
    import torch
    g = _assemble(c3.prob, c3.ad)
    I, J, V = _views(g)
    n = I.numel() - 1
    assert n == c3.ad.height and J.numel() == NNZ_C3 == int(I[-1])
    assert int(I[0]) == 0 and bool((I[1:] >= I[:-1]).all())
    rows = _rows(I)
    same = rows[1:] == rows[:-1]
    assert bool((J[1:][same] > J[:-1][same]).all())           # sorted, unique
    assert int((J.long() == rows).sum()) == n                 # one diagonal a row
    assert bool(torch.isfinite(torch.view_as_real(V)).all())
    V1 = V.clone()
    assert g.Assemble(True)
    assert torch.equal(torch.view_as_real(V), torch.view_as_real(V1))


def test_bloch_transpose(c3):
    import torch
    pm = copy.copy(c3.prob)
    pm.kx, pm.ky = -c3.prob.kx, -c3.prob.ky
    ga = _assemble(c3.prob, c3.ad, False)
    gb = _assemble(pm, c3.ad, False)
    Ia, Ja, Va = _views(ga)
    Ib, Jb, Vb = _views(gb)
    assert torch.equal(Ia, Ib) and torch.equal(Ja, Jb)        # symmetric pattern
    n = Ia.numel() - 1
    # A's entries in (column, row) order are A^T in CSR order
    perm = torch.argsort(Ja.long() * n + _rows(Ia))
    d = float((Va[perm] - Vb).abs().max() / Vb.abs().max())
    assert d < 1e-12, d
    assert float((Va - Vb).abs().max() / Vb.abs().max()) > 1e-6   # A itself is not symmetric


def test_linear_in_element_eps(c3):
    ad, prob = c3.ad, c3.prob
    e1 = configs.absorber_jitter(ad, prob, seed=101)
    e2 = configs.absorber_jitter(ad, prob, seed=202)
    vals = []
    for eps in (e1, e2, 0.5 * (e1 + e2)):
        pr = copy.copy(prob)
        pr.elem_eps = eps
        g = _assemble(pr, ad)
        vals.append(_views(g)[2].clone())
        g.Release()
    d = float((vals[0] + vals[1] - 2 * vals[2]).abs().max() / vals[2].abs().max())
    assert d < 1e-12, d


def test_spmv_matches_an_independent_product(c3):
    import torch
    g = _assemble(c3.prob, c3.ad)
    I, J, V = _views(g)
    n = I.numel() - 1
    gen = torch.Generator(device="cuda").manual_seed(7)
    x = torch.complex(torch.randn(n, generator=gen, device="cuda", dtype=torch.float64),
                      torch.randn(n, generator=gen, device="cuda", dtype=torch.float64))
    y = torch.empty_like(x)
    assert g.SpMV(x.data_ptr(), y.data_ptr())
    ref = torch.zeros_like(x).index_add_(0, _rows(I), V * x[J.long()])
    d = float((y - ref).abs().max() / ref.abs().max())
    assert d < 1e-13, d


def _element_sample(ad, elems):
    """The elements `elems` of ad as a mesh of their own: dofs renumbered
    densely in their original order, everything else as in ad."""
    ne, nd = len(elems), ad.nd
    dof = ad.dof.reshape(ad.ne, nd)[elems]
    used, inv = np.unique(dof, return_inverse=True)
    sub = dataclasses.replace(
        ad, ne=ne, height=len(used), dof=inv.reshape(-1).astype(ad.dof.dtype),
        sign=ad.sign.reshape(ad.ne, nd)[elems].reshape(-1),
        fo=(ad.fo.reshape(ad.ne, -1)[elems].reshape(-1) if ad.fo is not None and ad.fo.size
            else ad.fo),
        attr=ad.attr[elems], J=ad.J.reshape(ad.ne, 9)[elems].reshape(-1),
        Jinv=ad.Jinv.reshape(ad.ne, 9)[elems].reshape(-1), detJ=ad.detJ[elems],
        v0=ad.v0.reshape(ad.ne, 3)[elems].reshape(-1), I=None, Jcol=None,
        ess=np.searchsorted(used, np.intersect1d(ad.ess, used)).astype(ad.ess.dtype))
    sub.I, sub.Jcol = space.csr_symbolic(sub)
    return sub


def test_oracle_parity_on_a_sample_of_the_full_mesh(c3):
    ad, prob = c3.ad, c3.prob
    rng = np.random.default_rng(20260806)
    z = ad.v0.reshape(ad.ne, 3)[:, 2]
    pml = np.nonzero((z < np.quantile(z, 0.05)) | (z > np.quantile(z, 0.95)))[0]
    elems = np.unique(np.concatenate([rng.choice(ad.ne, 1200, replace=False),
                                      rng.choice(pml, 300, replace=False)]))
    sub = _element_sample(ad, elems)
    g = AsmGpuGlobal(prob)
    assert g.Init(sub, 0) and g.BuildGlobal(sub.ess)
    nb, npml = g.PathCounts()
    assert nb > 0 and npml > 0
    I, J = g.DownloadCsr()
    assert np.array_equal(I, sub.I) and np.array_equal(J, sub.Jcol)
    for elim in (True, False):
        assert g.Assemble(elim)
        want = oracle.assemble(sub, prob, sub.I, sub.Jcol, sub.ess, elim)
        d = float(np.abs(g.DownloadValues() - want).max() / np.abs(want).max())
        assert d < 1e-13, (elim, d)
