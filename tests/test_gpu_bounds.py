"""The bounds-checked debug build (liblfasm_bounds.so, device index checks
in the gather) on parity cases: no check fires and the values match the
oracle.  Runs in a child process because the library is loaded once per
process (LFASM_LIBRARY selects the build)."""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import os, sys, numpy as np
sys.path.insert(0, %(root)r)
from lithofem_b200 import _lib, configs
from lithofem_b200.asm import AsmGpuGlobal
from oracle import oracle
assert _lib.lib().lfasm_bounds_checked() == 1
cases = [configs.small_case("grating", 1, 6.0, seed=13, h=1.8),
         configs.small_case("hole", 2, 6.0, seed=13, h=2.4),
         configs.small_poly_case(3, 6.0, seed=5)]
for c in cases:
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
    I, J = oracle.csr(c.ad)
    for elim in (False, True):
        assert g.Assemble(elim), g.last_error
        ref = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, elim)
        r = np.abs(g.DownloadValues() - ref).max() / np.abs(ref).max()
        assert r < 1e-13, r
# the chunked assembly (many chunks) under the same checks
os.environ["LFASM_CHUNK_MB"] = "0.05"
c = configs.small_case("grating", 3, 6.0, seed=13, h=3.2)
g = AsmGpuGlobal(c.prob)
assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
I, J = oracle.csr(c.ad)
assert g.Assemble(True), g.last_error
ref = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, True)
assert np.abs(g.DownloadValues() - ref).max() / np.abs(ref).max() < 1e-13
print("bounds build ok")
"""


def test_bounds_checked_build_on_parity_cases():
    env = dict(os.environ, LFASM_LIBRARY=str(ROOT / "lithofem_b200" / "liblfasm_bounds.so"))
    out = subprocess.run([sys.executable, "-c", SCRIPT % {"root": str(ROOT)}], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "bounds build ok" in out.stdout


WAIT_SCRIPT = r"""
import os, sys, numpy as np
sys.path.insert(0, %(root)r)
from lithofem_b200 import _lib, configs
from lithofem_b200.asm import AsmGpuGlobal
from oracle import oracle
L = _lib.lib()
assert L.lfasm_bounds_checked() == 1
c = configs.small_case("grating", 3, 6.0, seed=13, h=3.2)
g = AsmGpuGlobal(c.prob)
assert g.Init(c.ad, 0) and g.SetPmlVariant(1) and g.BuildGlobal(c.ad.ess)
assert g.PathCounts()[1] > 0
# block 0's first chunk barrier never completes: the consumers' first wait
# there must run out after 4096 rounds and the call must report it
assert L.lfasm_debug_wait_test(0, 4096, 1) == 0
assert not g.Assemble(True)
assert "bounded wait ran out" in L.lfasm_last_error().decode(), L.lfasm_last_error()
# defaults back: the same handle assembles correctly on the same context
assert L.lfasm_debug_wait_test(0, 0, 0) == 0
I, J = oracle.csr(c.ad)
assert g.Assemble(True), g.last_error
ref = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, True)
r = np.abs(g.DownloadValues() - ref).max() / np.abs(ref).max()
assert r < 1e-13, r
print("wait run-out reported, device usable")
"""


def test_bounded_wait_runs_out_and_reports():
    """A bounded mbarrier wait of the warp-specialised PML kernel is made to
    run out (its producers withhold one barrier's arrivals, a debug-build
    injection); the assembly returns the error status, and the next
    assembly on the same context passes parity."""
    env = dict(os.environ, LFASM_LIBRARY=str(ROOT / "lithofem_b200" / "liblfasm_bounds.so"))
    out = subprocess.run([sys.executable, "-c", WAIT_SCRIPT % {"root": str(ROOT)}], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "wait run-out reported, device usable" in out.stdout
