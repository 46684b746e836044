"""Regenerate tests/golden/source_hole_p2_t6.npz from the REFERENCE's
scattered-field source.

Evaluates ScatterSource::Eval (solver/problem_common.inc:239-266, compiled
from the reference's sources into oracle/_ref/libref_asm.so) at every
mass-rule point of every element of a small seeded contact-hole mesh, p = 2,
theta = 6 deg, with the s and p plane-wave parts of lithofem_b200.incident
(themselves pinned to the reference by incident_golden.json).

    python tests/golden/make_source_golden.py
"""

from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from lithofem_b200 import configs, incident  # noqa: E402

FIXTURE = Path(__file__).resolve().parent / "source_hole_p2_t6.npz"


def case():
    return configs.small_case("hole", 2, 6.0, seed=21, h=2.4)


def parts(c):
    return [incident.planewave_parts(c.stack, c.theta, 0.0, pol, 1.0, True) for pol in ("s", "p")]


def digest(c) -> str:
    h = hashlib.sha256()
    for a in (c.ad.dof, c.ad.sign, c.ad.fo, c.ad.attr, c.ad.J, c.ad.v0, c.ad.rule_mass.ip):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main() -> None:
    from oracle import oracle
    c = case()
    f = oracle.ref_scatter_source(c.ad, c.prob, parts(c))
    np.savez_compressed(FIXTURE, digest=digest(c), f=f)
    print(FIXTURE, c.ad.ne, f.shape, int((np.abs(f).max(axis=(1, 2)) > 0).sum()), "source elements")


if __name__ == "__main__":
    main()
