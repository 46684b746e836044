"""Symmetric quadrature rules on the reference tetrahedron.

The reference tetrahedron is {x, y, z >= 0, x + y + z <= 1} with vertices
v0 = (0,0,0), v1 = (1,0,0), v2 = (0,1,0), v3 = (0,0,1); weights sum to its
volume 1/6.  Rules are stored as fully symmetric orbits in barycentric
coordinates (lambda0, lambda1, lambda2, lambda3) with reference coordinates
(x, y, z) = (lambda1, lambda2, lambda3).

The assembly path picks, per Nedelec order p, the rule of degree 2p - 2 for the
curl-curl term and of degree 2p for the mass and k-parallel terms (the
integrator defaults of the reference, solver/asm_data.inc:108-116).  The point
counts (1, 4, 11, 24 for degree 0, 2, 4, 6) are those of the classic Keast
symmetric rules; the orbit parameters below were produced by moment fitting
(``quadrature_fit.py``) and every rule is exact for all polynomials of its
degree (checked in tests/test_basis.py).
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass
from functools import lru_cache

import numpy as np

# degree -> list of (orbit kind, parameters..., weight) ; strings keep 25 digits
RULE_ORBITS: dict[int, list[tuple]] = {
    0: [("S4", "0.1666666666666666666666667")],
    2: [("S31", "0.1381966011250105151795413", "0.04166666666666666666666667")],
    4: [
        ("S4", "-0.01315555555555555555555556"),
        ("S31", "0.07142857142857142857142857", "0.007622222222222222222222222"),
        ("S22", "0.1005964238332007950038979", "0.02488888888888888888888889"),
    ],
    6: [
        ("S31", "0.2146028712591520292888392", "0.006653791709694582016615105"),
        ("S31", "0.04067395853461135311557945", "0.001679535175886773824668873"),
        ("S31", "0.3223378901422755103439945", "0.009226196923942453682525546"),
        ("S211", "0.06366100187501752529923553", "0.6030056647916491413674311",
         "0.008035714285714285714285714"),
    ],
}


def _orbit_points(kind: str, par: list[float]) -> list[tuple[float, ...]]:
    if kind == "S4":
        base = (0.25, 0.25, 0.25, 0.25)
    elif kind == "S31":
        a = par[0]
        base = (a, a, a, 1.0 - 3.0 * a)
    elif kind == "S22":
        a = par[0]
        base = (a, a, 0.5 - a, 0.5 - a)
    elif kind == "S211":
        a, b = par
        base = (a, a, b, 1.0 - 2.0 * a - b)
    else:  # pragma: no cover - table is fixed
        raise ValueError(kind)
    out: list[tuple[float, ...]] = []
    for perm in itertools.permutations(range(4)):
        p = tuple(base[i] for i in perm)
        if p not in out:
            out.append(p)
    return out


@dataclass(frozen=True)
class TetRule:
    """Quadrature rule: ``ip`` (nq, 3) reference coordinates, ``w`` (nq,)."""

    degree: int
    ip: np.ndarray
    w: np.ndarray

    @property
    def nq(self) -> int:
        return int(self.w.shape[0])


@lru_cache(maxsize=None)
def tet_rule(degree: int) -> TetRule:
    """Lowest tabulated symmetric rule exact to at least ``degree``."""
    degree = max(0, int(degree))
    avail = sorted(RULE_ORBITS)
    use = next((d for d in avail if d >= degree), None)
    if use is None:
        raise ValueError(f"no tetrahedron rule of degree {degree} (max {avail[-1]})")
    pts: list[tuple[float, ...]] = []
    wts: list[float] = []
    for orb in RULE_ORBITS[use]:
        kind = orb[0]
        vals = [float(s) for s in orb[1:]]
        par, w = vals[:-1], vals[-1]
        for p in _orbit_points(kind, par):
            pts.append(p)
            wts.append(w)
    lam = np.array(pts, dtype=np.float64)
    ip = np.ascontiguousarray(lam[:, 1:4])
    return TetRule(degree=use, ip=ip, w=np.array(wts, dtype=np.float64))
