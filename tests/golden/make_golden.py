"""Regenerate the golden fixtures from the REFERENCE's own assembly code.

Runs the reference reassembler compiled from its sources (oracle/_ref,
built by `make -C oracle` where the reference tree exists) on tiny seeded
meshes of the three benchmark geometries and stores, per case, a digest of
the inputs, the reference symbolic CSR (build_csr_symbolic: the row pointer
in full, a SHA-256 of the column array), the values (reassemble_all) as an
every-STRIDE-th subsample plus three full-array checksums, and two element
matrices (reassemble_element) in full.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from lithofem_b200 import configs  # noqa: E402
from oracle import oracle  # noqa: E402

CASES = [("slab", 1, 0.0), ("slab", 2, 6.0), ("hole", 1, 6.0), ("hole", 2, 0.0),
         ("grating", 2, 6.0), ("grating", 3, 6.0), ("hole", 3, 0.0)]
H = {1: 2.4, 2: 3.0, 3: 4.0}
STRIDE = 17


def checksums(vals: np.ndarray) -> np.ndarray:
    k = np.arange(len(vals), dtype=np.float64)
    w = np.cos(0.37 * k) + 0.5
    return np.array([vals.sum(), (np.abs(vals) ** 2).sum() + 0j, (w * vals).sum()])


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


def digest(ad) -> str:
    h = hashlib.sha256()
    for a in (ad.dof, ad.sign, ad.fo, ad.attr, ad.J, ad.detJ, ad.v0, ad.rule_cc.curl,
              ad.rule_mass.vshape):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case_of(kind, p, theta):
    return configs.small_case(kind, p, theta, seed=11, h=H[p])


def main() -> None:
    out = Path(__file__).resolve().parent
    for kind, p, theta in CASES:
        c = case_of(kind, p, theta)
        rc = oracle.RefContext(c.ad, c.prob)
        I, J = rc.build_csr()
        vals = rc.reassemble()
        els = np.array([0, c.ad.ne - 1])
        elm = np.stack([rc.element(int(e)) for e in els])
        name = f"ref_{kind}_p{p}_t{int(theta)}.npz"
        np.savez_compressed(out / name, digest=digest(c.ad), I=I, J_sha=sha(J), nnz=len(J),
                            vals_sub=vals[::STRIDE], checksums=checksums(vals),
                            elements=els, element_mats=elm)
        print(name, c.ad.ne, c.ad.height, len(J))


if __name__ == "__main__":
    main()
