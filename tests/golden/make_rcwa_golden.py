"""Regenerate tests/golden/rcwa_golden.json from the REFERENCE's RCWA module.

Imports tests/reference/rcwa.py from the reference tree (numpy/scipy only),
the grating oracle of the reference's line-grating tests
(tests/test_solver_m8.py:96-143), and records the order efficiencies of
its propagating orders for:

* absorber line gratings in vacuum (TE and TM, two duty cycles) on a
  20 nm period, 6 nm high cell -- the reference's 48 nm / 40 nm cell scaled
  down so that a host LU of the assembled system ends in seconds;
* a uniform absorber layer (duty 1), TE and TM, which must equal the
  transfer-matrix result (the reference's tests/test_rcwa_selfcheck.py).

    python tests/golden/make_rcwa_golden.py
"""

from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

REF = Path("/root/reference/tests/reference/rcwa.py")
OUT = Path(__file__).with_name("rcwa_golden.json")
ABS = complex(0.95, 0.031) ** 2          # absorber n, k = 0.95, 0.031
WAVELENGTH, THETA = 13.5, 6.0
PERIOD, HEIGHT, N_ORDERS = 20.0, 6.0, 101

CASES = [
    # (name, duty, pol)
    ("line_d50_te", 0.5, "TE"),
    ("line_d50_tm", 0.5, "TM"),
    ("line_d25_te", 0.25, "TE"),
    ("line_d25_tm", 0.25, "TM"),
    ("uniform_te", 1.0, "TE"),
    ("uniform_tm", 1.0, "TM"),
]


def load_ref():
    spec = importlib.util.spec_from_file_location("ref_rcwa", REF)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ref_rcwa"] = mod
    spec.loader.exec_module(mod)
    return mod


def main() -> None:
    rcwa = load_ref()
    out = {"source": "tests/reference/rcwa.py", "period": PERIOD, "height": HEIGHT,
           "wavelength": WAVELENGTH, "theta": THETA, "eps_line": [ABS.real, ABS.imag],
           "n_orders": N_ORDERS, "cases": {}}
    for name, duty, pol in CASES:
        if duty >= 1.0:
            layer = rcwa.Layer(HEIGHT, (1.0,), (ABS,))
        else:
            layer = rcwa.Layer(HEIGHT, (duty, 1.0 - duty), (ABS, 1.0 + 0j))
        res = rcwa.solve(PERIOD, WAVELENGTH, THETA, pol, [layer], 1.0, 1.0, n_orders=N_ORDERS)
        prop = np.abs(res.qz_in.imag) < 1e-12
        out["cases"][name] = {
            "duty": duty, "pol": pol,
            "orders": [int(m) for m in res.orders[prop]],
            "r_eff": [float(e) for e in res.r_eff[prop]],
            "t_eff": [float(e) for e in res.t_eff[prop]],
        }
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
