"""Scattered-field RHS pinned to the reference's source term.

The reference forms its RHS source with ScatterSource::Eval and incident_at
(solver/problem_common.inc:219-266) and integrates it with MFEM's
VectorFEDomainLFIntegrator (lithofem_solve.cpp:678-684).  Here:

* ``incident_at`` of the reference (compiled from its sources, oracle/_ref)
  equals the table evaluation of lithofem_b200.incident on the same tables;
* the reference's ScatterSource values at every mass-rule point, integrated
  by tests/ref_rhs.py, equal the oracle's RHS (oracle.rhs), which the GPU
  RHS is compared with in the GPU parity tests;
* a committed fixture of reference source values (made by
  tests/golden/make_source_golden.py) pins the same without the shim.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from lithofem_b200 import configs, incident
from oracle import oracle

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from ref_rhs import rhs_from_points  # noqa: E402
import make_source_golden as SG  # noqa: E402

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference shim not built")
CASES = [("hole", 2, 6.0), ("grating", 3, 6.0), ("hole", 1, 6.0), ("grating", 2, 0.0)]


def _parts(c, pols=("s", "p")):
    return [incident.planewave_parts(c.stack, c.theta, 0.0, pol, 1.0, True) for pol in pols]


@needs_ref
def test_reference_incident_at_equals_table_evaluation():
    c = configs.small_case("grating", 2, 6.0, seed=3)
    parts = _parts(c)
    oracle.ref_set_problem(c.prob, c.p)
    oracle.ref_set_incident(parts)
    rng = np.random.default_rng(1)
    for s, sw in enumerate(parts[0]):
        for z in rng.uniform(sw.z_lo, sw.z_hi, 7):
            want = oracle.ref_incident_at(s, z)
            got = incident.eval_parts(parts, np.array([z]))[0]
            assert np.abs(got - want).max() <= 1e-14 * max(1.0, np.abs(want).max())


@needs_ref
@pytest.mark.parametrize("kcase", CASES, ids=[f"{k}-p{p}-t{t:g}" for k, p, t in CASES])
def test_oracle_rhs_equals_reference_source(kcase):
    c = configs.small_case(*kcase, seed=5)
    parts = _parts(c)
    f = oracle.ref_scatter_source(c.ad, c.prob, parts)
    assert np.abs(f).max() > 0, "no frustum element in the case"
    want = rhs_from_points(c.ad, f, c.ad.ess, True)
    got = oracle.rhs(c.ad, c.prob, parts, [0, 0], 1, c.ad.ess, True)[0]
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_oracle_rhs_equals_reference_source_fixture():
    g = np.load(SG.FIXTURE)
    c = SG.case()
    assert SG.digest(c) == str(g["digest"]), "inputs drifted from the fixture"
    parts = SG.parts(c)
    want = rhs_from_points(c.ad, g["f"], c.ad.ess, True)
    got = oracle.rhs(c.ad, c.prob, parts, [0, 0], 1, c.ad.ess, True)[0]
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
