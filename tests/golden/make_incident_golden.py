"""Regenerate tests/golden/incident_golden.json from the REFERENCE's
incident-field construction.

Imports src/lithofem/incident.py (with its tmm and constants modules) from
the reference tree.  Its ``config`` import needs shapely, which is absent,
so a stand-in module providing the three names incident.py imports
(Model, PlaneWave, SolveGroup) is registered first; _planewave_field
(src/lithofem/incident.py:121-205) reads only model.wavelength,
model.slabs, model.eps_bg_of_slab and the plane wave's theta, phi,
from_top and kpar, which the stand-ins carry.  The recorded per-slab tables
(z range, qA, zA, A, qB, zB, B) pin lithofem_b200.incident.planewave_parts.

    python tests/golden/make_incident_golden.py
"""

from __future__ import annotations

import importlib.util
import json
import math
import sys
import types
from dataclasses import dataclass
from pathlib import Path

import numpy as np

REF = Path("/root/reference/src/lithofem")
ABS = complex(0.95, 0.031) ** 2
UND = complex(0.97, 0.01) ** 2

# (name, wavelength, slab breakpoints, background eps per slab)
STACKS = [
    ("absorber slab", 13.5, [0.0, 60.0, 120.0], [ABS, 1.0]),
    ("grating absorber over underlayer", 13.5, [0.0, 40.0, 100.0, 130.0], [UND, ABS, 1.0]),
    ("three layers", 193.0, [-20.0, 15.0, 52.0, 110.0, 140.0],
     [1.5 ** 2, 1.2 ** 2 + 0.01j, 2.0 ** 2, 1.0]),
]
WAVES = [  # (theta, phi, pol, from_top, amplitude)
    (0.0, 0.0, "s", True, 1.0),
    (0.0, 0.0, "p", True, 1.0),
    (6.0, 0.0, "s", True, 1.0),
    (6.0, 0.0, "p", True, 1.0),
    (6.0, 30.0, "s", True, 0.6 + 0.8j),
    (6.0, 30.0, "p", True, 0.6 - 0.8j),
    (12.0, 0.0, "s", False, 1.0),
    (12.0, 45.0, "p", False, 1.0),
]


def load_ref():
    pkg = types.ModuleType("lithofem")
    pkg.__path__ = [str(REF)]
    sys.modules["lithofem"] = pkg
    cfg = types.ModuleType("lithofem.config")

    @dataclass(frozen=True)
    class PlaneWave:
        theta: float
        phi: float
        from_top: bool
        kpar: tuple

    class Model:  # only the attributes _planewave_field reads
        pass

    class SolveGroup:
        pass

    cfg.Model, cfg.PlaneWave, cfg.SolveGroup = Model, PlaneWave, SolveGroup
    sys.modules["lithofem.config"] = cfg
    mods = {}
    for name in ("constants", "tmm", "incident"):
        spec = importlib.util.spec_from_file_location(f"lithofem.{name}", REF / f"{name}.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[f"lithofem.{name}"] = mod
        spec.loader.exec_module(mod)
        mods[name] = mod
    return mods, PlaneWave


class _Model:
    def __init__(self, wavelength, slabs, eps):
        self.wavelength, self.slabs, self._eps = wavelength, list(slabs), list(eps)

    def eps_bg_of_slab(self, i):
        return complex(self._eps[i])


def c2(z):
    return [complex(z).real, complex(z).imag]


def main() -> None:
    mods, PlaneWave = load_ref()
    inc, const = mods["incident"], mods["constants"]
    out = []
    for sname, wl, slabs, eps in STACKS:
        model = _Model(wl, slabs, eps)
        for th, ph, pol, top, amp in WAVES:
            kk = const.k0(wl) * np.sin(np.deg2rad(th))
            kpar = (kk * float(np.cos(np.deg2rad(ph))), kk * float(np.sin(np.deg2rad(ph))))
            pw = PlaneWave(theta=th, phi=ph, from_top=top, kpar=kpar)
            part = inc._planewave_field(model, pw, pol, amp)
            out.append({
                "stack": sname, "wavelength": wl, "slabs": slabs, "eps": [c2(e) for e in eps],
                "theta": th, "phi": ph, "pol": pol, "from_top": top, "amp": c2(amp),
                "r_amp": c2(part.r_amp), "t_amp": c2(part.t_amp),
                "tables": [{"z": [sw.z_lo, sw.z_hi], "qA": c2(sw.qA), "zA": sw.zA,
                            "A": [c2(v) for v in sw.A], "qB": c2(sw.qB), "zB": sw.zB,
                            "B": [c2(v) for v in sw.B]} for sw in part.slabs]})
    p = Path(__file__).resolve().parent / "incident_golden.json"
    p.write_text(json.dumps(out, indent=0))
    print(p, len(out), "cases")
    assert math.isfinite(out[0]["r_amp"][0])


if __name__ == "__main__":
    main()
