"""Regenerate tests/golden/tmm_golden.json from the REFERENCE's TMM module.

Imports src/lithofem/tmm.py from the reference tree (numpy only) and records
r, t and the per-layer q, a, b for a set of stacks, angles and
polarisations, including the absorber/underlayer stacks of the benchmarks.

    python tests/golden/make_tmm_golden.py
"""

from __future__ import annotations

import importlib.util
import json
import math
from pathlib import Path

REF = Path("/root/reference/src/lithofem/tmm.py")
ABS = complex(0.95, 0.031) ** 2
UND = complex(0.97, 0.01) ** 2


def load_ref():
    import sys
    import types
    pkg = types.ModuleType("lithofem")
    pkg.__path__ = [str(REF.parent)]
    sys.modules.setdefault("lithofem", pkg)
    spec = importlib.util.spec_from_file_location("lithofem.constants", REF.parent / "constants.py")
    const = importlib.util.module_from_spec(spec)
    sys.modules["lithofem.constants"] = const
    spec.loader.exec_module(const)
    spec = importlib.util.spec_from_file_location("lithofem.tmm", REF)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lithofem.tmm"] = mod
    spec.loader.exec_module(mod)
    return mod


CASES = [
    # (eps_in, eps_out, eps layers, d layers, wavelength, theta, pol)
    (1.0, 2.25, [], [], 500.0, 0.0, "s"),
    (1.0, 2.25, [], [], 500.0, 30.0, "p"),
    (1.0, ABS, [ABS], [60.0], 13.5, 0.0, "s"),
    (1.0, ABS, [1.0, ABS], [60.0, 60.0], 13.5, 6.0, "s"),
    (1.0, ABS, [1.0, ABS], [60.0, 60.0], 13.5, 6.0, "p"),
    (1.0, UND, [1.0, 1.0, UND], [30.0, 60.0, 40.0], 13.5, 6.0, "s"),
    (1.0, UND, [1.0, 1.0, UND], [30.0, 60.0, 40.0], 13.5, 6.0, "p"),
    (1.0, 1.5 ** 2, [1.2 ** 2 + 0.01j, 2.0 ** 2], [100.0, 37.0], 193.0, 45.0, "p"),
]


def c2(z):
    return [complex(z).real, complex(z).imag]


def main() -> None:
    tm = load_ref()
    out = []
    for ein, eout, eps, d, wl, th, pol in CASES:
        st = tm.Stack(eps_in=ein, eps_out=eout, eps=tuple(eps), d=tuple(d))
        r = tm.solve(st, wl, theta_deg=th, pol=pol)
        out.append({"eps_in": c2(ein), "eps_out": c2(eout), "eps": [c2(e) for e in eps],
                    "d": d, "wavelength": wl, "theta": th, "pol": pol,
                    "r": c2(r.r), "t": c2(r.t), "q": [c2(v) for v in r.q],
                    "a": [c2(v) for v in r.a], "b": [c2(v) for v in r.b]})
    p = Path(__file__).resolve().parent / "tmm_golden.json"
    p.write_text(json.dumps(out, indent=1))
    print(p, len(out))


if __name__ == "__main__":
    main()
