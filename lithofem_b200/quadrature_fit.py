"""Generator for the symmetric tetrahedron quadrature rules in ``quadrature.py``.

Run ``python -m lithofem_b200.quadrature_fit`` to regenerate the orbit
parameters printed into ``quadrature.RULE_ORBITS``.  Not imported by the
library at run time (it needs mpmath).

Method: moment fitting with fully symmetric orbits (Keast-type structure).
Points are parametrised in barycentric coordinates by S4-orbits

* ``S4``           (1/4, 1/4, 1/4, 1/4)                    1 point
* ``S31(a)``       (a, a, a, 1-3a)                          4 points
* ``S22(a)``       (a, a, 1/2-a, 1/2-a)                     6 points
* ``S211(a, b)``   (a, a, b, 1-2a-b)                       12 points

and the unknown (parameters, weight) per orbit are fixed by requiring the
rule to integrate exactly every S4-invariant polynomial of degree <= d on
the reference tetrahedron {x, y, z >= 0, x + y + z <= 1} (volume 1/6).
The invariant ring on the simplex is generated by the power sums
p2, p3, p4 of the barycentric coordinates, so the moment equations are
the products p2^i p3^j p4^k with 2i + 3j + 4k <= d.  The exact integral of
a barycentric monomial is |T| 3! a! b! c! e! / (a + b + c + e + 3)!.  The
square nonlinear system is solved by Newton's method in 40-digit
arithmetic from a rough starting guess.
"""

from __future__ import annotations

import itertools
from math import factorial

import mpmath as mp

mp.mp.dps = 40

NPAR = {"S4": 0, "S31": 1, "S22": 1, "S211": 2}


def _orbit(kind, par):
    if kind == "S4":
        base = (mp.mpf(1) / 4,) * 4
    elif kind == "S31":
        a = par[0]
        base = (a, a, a, 1 - 3 * a)
    elif kind == "S22":
        a = par[0]
        base = (a, a, mp.mpf(1) / 2 - a, mp.mpf(1) / 2 - a)
    else:
        a, b = par
        base = (a, a, b, 1 - 2 * a - b)
    pts = {}
    for perm in itertools.permutations(range(4)):
        key = tuple(int(perm[i]) for i in range(4))
        pts[tuple(base[i] for i in key)] = None
    # dedupe numerically-equal permutations (exact for mp values)
    uniq = []
    for p in pts:
        if not any(all(p[i] == q[i] for i in range(4)) for q in uniq):
            uniq.append(p)
    return uniq


def _exact_mono(alpha):
    num = 1
    for a in alpha:
        num *= factorial(a)
    return mp.mpf(num) * 6 / factorial(sum(alpha) + 3) / 6


def _invariants(deg):
    return [(i, j, k) for i in range(deg // 2 + 1) for j in range(deg // 3 + 1)
            for k in range(deg // 4 + 1) if 2 * i + 3 * j + 4 * k <= deg]


def _inv_exact(ijk):
    i, j, k = ijk
    poly = {(0, 0, 0, 0): 1}

    def mul(P, Q):
        R = {}
        for a, ca in P.items():
            for b, cb in Q.items():
                e = tuple(x + y for x, y in zip(a, b))
                R[e] = R.get(e, 0) + ca * cb
        return R

    def pk(kk):
        return {tuple(kk if t == s else 0 for t in range(4)): 1 for s in range(4)}

    for _ in range(i):
        poly = mul(poly, pk(2))
    for _ in range(j):
        poly = mul(poly, pk(3))
    for _ in range(k):
        poly = mul(poly, pk(4))
    return sum(c * _exact_mono(e) for e, c in poly.items())


def fit(structure, deg, x0):
    invs = _invariants(deg)
    ex = [_inv_exact(t) for t in invs]

    def residual(*x):
        out = [mp.mpf(0)] * len(invs)
        o = 0
        for kind in structure:
            n = NPAR[kind]
            par = x[o:o + n]
            w = x[o + n]
            o += n + 1
            for p in _orbit(kind, par):
                p2 = sum(v ** 2 for v in p)
                p3 = sum(v ** 3 for v in p)
                p4 = sum(v ** 4 for v in p)
                for r, (i, j, k) in enumerate(invs):
                    out[r] += w * p2 ** i * p3 ** j * p4 ** k
        return [o_ - e for o_, e in zip(out, ex)]

    assert len(invs) == len(x0), (len(invs), len(x0))
    return mp.findroot(residual, [mp.mpf(v) for v in x0])


START = {
    0: (["S4"], [1.0 / 6]),
    2: (["S31"], [0.138, 0.04]),
    4: (["S4", "S31", "S22"], [-0.0132, 0.0714, 0.0076, 0.1006, 0.0249]),
    6: (["S31", "S31", "S31", "S211"],
        [0.2146, 0.0066, 0.0407, 0.0017, 0.3223, 0.0092, 0.0637, 0.6030, 0.0080]),
}


def main() -> None:
    for deg, (structure, x0) in START.items():
        if deg == 0:
            print(deg, structure, ["0.16666666666666666666666666666666666667"])
            continue
        x = fit(structure, deg, x0)
        print(deg, structure, [mp.nstr(v, 25) for v in x])


if __name__ == "__main__":
    main()
