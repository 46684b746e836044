"""The drop-in call site of INTEGRATION.md section 2 (gpu_assemble, which
replaces AsmGpu / AsmGpuGlobal at solver/lithofem_solve.cpp:765-795),
compiled against the reference's own AsmData, Region and Problem.

* CPU: the document's first C++ block, extracted as oracle/Makefile does,
  compiles with nvcc against the reference's headers and the shim
  (oracle/ref_shim/dropin.cu), so a field-order or type slip in the
  documented call site fails here.
* GPU: the compiled call site assembles the same CSR, bit for bit, as the
  Python (ctypes) path on the same inputs.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

ROOT = Path(__file__).resolve().parents[1]
REF_SOLVER = Path("/root/reference/solver")


@pytest.mark.skipif(not (REF_SOLVER / "asm_data.inc").exists() or not shutil.which("nvcc"),
                    reason="reference tree or nvcc not present")
def test_documented_call_site_compiles(tmp_path):
    text = (ROOT / "INTEGRATION.md").read_text().splitlines()
    start = text.index("```cpp") + 1
    end = start + text[start:].index("```")
    (tmp_path / "dropin_snippet.inc").write_text("\n".join(text[start:end]) + "\n")
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c",
           "-I", str(ROOT / "oracle" / "ref_shim"), "-I", str(REF_SOLVER), "-I", str(tmp_path),
           "-I", str(ROOT / "include"), "-o", str(tmp_path / "dropin.o"),
           str(ROOT / "oracle" / "ref_shim" / "dropin.cu")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.dropin_available(), reason="drop-in call site not built")
@pytest.mark.parametrize("kcase", [("grating", 3, 6.0), ("hole", 2, 6.0), ("slab", 1, 0.0)],
                         ids=["grating-p3", "hole-p2", "slab-p1"])
def test_call_site_equals_ctypes_path(kcase):
    from lithofem_b200 import configs
    from lithofem_b200.asm import AsmGpuGlobal
    c = configs.small_case(*kcase, seed=13)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess) and g.Assemble(True)
    I, J = g.DownloadCsr()
    V = g.DownloadValues()
    g.Release()
    Id, Jd, Vd = oracle.dropin_assemble(c.ad, c.prob)
    assert np.array_equal(I, Id) and np.array_equal(J, Jd)
    assert np.array_equal(V.view(np.float64), Vd.view(np.float64)), \
        float(np.abs(V - Vd).max() / np.abs(V).max())
