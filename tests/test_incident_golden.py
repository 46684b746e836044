"""Incident-field tables against the reference's own construction.

tests/golden/incident_golden.json holds the per-slab tables that the
reference's _planewave_field (src/lithofem/incident.py:121-205) builds for
three stacks, normal and oblique incidence, s and p, from the top and from
the bottom, real and complex amplitudes (made by make_incident_golden.py,
which imports the reference module).  ``incident.planewave_parts`` must
reproduce every table: the phase references zA/zB exactly, the wavenumbers
and vector amplitudes to rounding.
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from lithofem_b200 import incident

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "incident_golden.json").read_text())


def _c(v):
    return complex(v[0], v[1])


class _Stack:
    """The three attributes planewave_parts reads from a layer stack."""

    def __init__(self, g):
        self.wavelength = g["wavelength"]
        self.slabs = list(g["slabs"])
        self._eps = [_c(e) for e in g["eps"]]

    @property
    def k0(self):
        return 2.0 * math.pi / self.wavelength

    def eps_bg_of_slab(self, i):
        return self._eps[i]


@pytest.mark.parametrize("g", GOLD, ids=[f"{g['stack'][:8]}-{g['pol']}{g['theta']:g}-{g['phi']:g}-"
                                         f"{'top' if g['from_top'] else 'bot'}" for g in GOLD])
def test_planewave_tables_match_reference(g):
    parts = incident.planewave_parts(_Stack(g), g["theta"], g["phi"], g["pol"], _c(g["amp"]),
                                     g["from_top"])
    assert len(parts) == len(g["tables"])
    scale = max(max(abs(_c(v)) for v in t["A"] + t["B"]) for t in g["tables"])
    for sw, t in zip(parts, g["tables"]):
        assert (sw.z_lo, sw.z_hi) == tuple(t["z"])
        assert abs(sw.zA - t["zA"]) <= 1e-12 * max(1.0, abs(t["zA"]))
        assert abs(sw.zB - t["zB"]) <= 1e-12 * max(1.0, abs(t["zB"]))
        for q, key in ((sw.qA, "qA"), (sw.qB, "qB")):
            assert abs(q - _c(t[key])) <= 1e-13 * abs(_c(t[key])) + 1e-15
        for vec, key in ((sw.A, "A"), (sw.B, "B")):
            ref = np.array([_c(v) for v in t[key]])
            assert np.abs(np.asarray(vec) - ref).max() <= 1e-12 * scale


def test_table_evaluation_is_continuous_across_slabs():
    """The summed tables give one continuous tangential field across every
    slab face (the property the RHS relies on), for the recorded cases."""
    for g in GOLD:
        parts = incident.planewave_parts(_Stack(g), g["theta"], g["phi"], g["pol"],
                                         _c(g["amp"]), g["from_top"])
        for i in range(len(parts) - 1):
            z = parts[i].z_hi
            lo = parts[i].eval(z)[0]
            hi = parts[i + 1].eval(z)[0]
            assert np.abs(lo[:2] - hi[:2]).max() <= 1e-11 * max(1.0, np.abs(lo).max())
