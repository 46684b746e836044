"""C ABI: the in-tree library loads and exports every declared entry point
(no device work: runs without a GPU)."""

from __future__ import annotations

import ctypes as ct

import numpy as np

from lithofem_b200 import _abi, _lib, configs


def test_library_exports_every_header_symbol():
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_header_structs_match_ctypes_layout():
    # pointer-size sanity of the mirrored structs
    assert ct.sizeof(_abi.RefRule) == 8 + 4 * 8
    assert _abi.AsmDataC.rule_cc.offset % 8 == 0


def test_argument_validation_precedes_device_use():
    c = configs.small_case("slab", 1, 0.0)
    m = _abi.marshal(c.ad, c.prob)
    m.ad.ne = 0
    h = ct.c_void_p()
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 1 and b"empty mesh" in _lib.lib().lfasm_last_error()
    m = _abi.marshal(c.ad, c.prob)
    m.ad.p = 4
    m.ad.nd = 84
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 3
    bad = c.ad.dof.copy()
    bad[5] = c.ad.height
    keep = np.ascontiguousarray(bad, dtype=np.int32)
    m = _abi.marshal(c.ad, c.prob)
    m.ad.dof = keep.ctypes.data_as(_abi.c_int_p)
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 1 and b"out of range" in _lib.lib().lfasm_last_error()


def _init_with(c, **arrays):
    m = _abi.marshal(c.ad, c.prob)
    keep = []
    for name, arr in arrays.items():
        a = np.ascontiguousarray(arr)
        keep.append(a)
        ptr_t = _abi.c_int_p if a.dtype == np.int32 else _abi.c_double_p
        setattr(m.ad, name, a.ctypes.data_as(ptr_t))
    h = ct.c_void_p()
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    return rc, _lib.lib().lfasm_last_error().decode()


def test_validation_reports_the_first_offending_entry():
    """Each check names the lowest bad index, checks run in the order dof,
    then per element attr before detJ, then face orientations -- all before
    any device call."""
    c = configs.small_case("grating", 2, 6.0)
    dof = c.ad.dof.astype(np.int32).copy()
    dof[[40000 % dof.size, 9000 % dof.size, 77]] = -3
    rc, msg = _init_with(c, dof=dof)
    assert rc == 1 and msg.startswith("dof[77] = -3 out of range")
    attr = c.ad.attr.astype(np.int32).copy()
    attr[[50, 20]] = len(c.prob.regions) + 1
    detJ = c.ad.detJ.copy()
    detJ[[30, 7]] = [np.nan, -1.0]
    rc, msg = _init_with(c, attr=attr)
    assert rc == 1 and msg.startswith("attr[20] =")
    rc, msg = _init_with(c, detJ=detJ)
    assert rc == 1 and msg == "detJ[7] not positive"
    rc, msg = _init_with(c, attr=attr, detJ=detJ)   # element 7 is checked before 20
    assert rc == 1 and msg == "detJ[7] not positive"
    attr2 = attr.copy()
    attr2[7] = 0
    rc, msg = _init_with(c, attr=attr2, detJ=detJ)  # attr before detJ on one element
    assert rc == 1 and msg.startswith("attr[7] = 0")
    fo = c.ad.fo.astype(np.int32).copy()
    fo[[11, 3]] = [6, -1]
    rc, msg = _init_with(c, fo=fo)
    assert rc == 1 and msg == "fo[3] = -1 outside 0..5"


def test_injected_failure(monkeypatch, capfd):
    """LITHOFEM_ASM_FORCE_FAIL (the reference's host-side switch,
    solver/lithofem_solve.cpp:757-762) makes lfasm_init fail before any
    other work, with the reference's log line."""
    c = configs.small_case("slab", 1, 0.0)
    m = _abi.marshal(c.ad, c.prob)
    h = ct.c_void_p()
    monkeypatch.setenv("LITHOFEM_ASM_FORCE_FAIL", "1")
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 6 and not h.value
    assert b"LITHOFEM_ASM_FORCE_FAIL" in _lib.lib().lfasm_last_error()
    assert "asm_gpu: forced failure injected (LITHOFEM_ASM_FORCE_FAIL)" in capfd.readouterr().out


def test_bounds_checked_build_loads():
    """The debug build with device index checks exports the same entry
    points and reports itself; the production build reports 0."""
    from pathlib import Path
    dbg = Path(_lib.__file__).resolve().parent / "liblfasm_bounds.so"
    L = ct.CDLL(str(dbg))
    for name in _lib.exported_symbols():
        assert hasattr(L, name), name
    assert L.lfasm_bounds_checked() == 1
    assert _lib.lib().lfasm_bounds_checked() == 0


def test_validation_of_large_arrays_reports_the_lowest_index():
    """Arrays above a million entries are scanned by several host threads;
    the message still names the lowest offending entry."""
    c = configs.small_case("slab", 1, 0.0)
    ne = 400_000
    nd = c.ad.nd
    reps = -(-ne // c.ad.ne)
    dof = np.tile(c.ad.dof.reshape(c.ad.ne, nd), (reps, 1))[:ne].reshape(-1).astype(np.int32)
    attr = np.tile(c.ad.attr, reps)[:ne].astype(np.int32)
    detJ = np.tile(c.ad.detJ, reps)[:ne].copy()
    bad = dof.copy()
    bad[[2_100_000, 1_900_000, 1_400_001]] = -1
    m = _abi.marshal(c.ad, c.prob)
    m.ad.ne = ne
    keep = [bad, attr, detJ]
    m.ad.dof = bad.ctypes.data_as(_abi.c_int_p)
    m.ad.attr = attr.ctypes.data_as(_abi.c_int_p)
    m.ad.detJ = detJ.ctypes.data_as(_abi.c_double_p)
    h = ct.c_void_p()
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 1 and _lib.lib().lfasm_last_error().startswith(b"dof[1400001] = -1")
    detJ[[399_000, 250_001]] = 0.0
    m.ad.dof = dof.ctypes.data_as(_abi.c_int_p)
    rc = _lib.lib().lfasm_init(ct.byref(m.ad), ct.byref(m.prob), 0, ct.byref(h))
    assert rc == 1 and _lib.lib().lfasm_last_error() == b"detJ[250001] not positive"
    del keep


def test_tuning_entry_points_reject_a_null_handle():
    """The variant setters and getters check their handle before anything
    else; the header's variant count is the one the Python layer sizes its
    buffers with."""
    import re
    from pathlib import Path
    L = _lib.lib()
    null = ct.c_void_p()
    v = ct.c_int()
    ms = (ct.c_float * _abi.BULK_VARIANTS)()
    for rc in (L.lfasm_set_bulk_variant(null, 1), L.lfasm_set_pml_variant(null, 1),
               L.lfasm_get_tuning(null, ct.byref(v), ms),
               L.lfasm_get_pml_tuning(null, ct.byref(v), ms), L.lfasm_autotune(null)):
        assert rc == 1 and b"NULL handle" in L.lfasm_last_error()
    header = (Path(__file__).resolve().parents[1] / "include" / "lfasm.h").read_text()
    n = int(re.search(r"#define LFASM_BULK_VARIANTS (\d+)", header).group(1))
    assert n == _abi.BULK_VARIANTS == 6


def test_no_cpu_fallback(tmp_path):
    """Without its library the Python layer raises on first use; with the
    library but without a usable GPU, lfasm_init fails with a CUDA error
    instead of computing anything on the host."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = ("from lithofem_b200 import configs\n"
            "from lithofem_b200.asm import AsmGpu\n"
            "c = configs.small_case('slab', 1, 0.0)\n"
            "g = AsmGpu(c.prob)\n"
            "try:\n"
            "    ok = g.Init(c.ad, 0)\n"
            "except RuntimeError as e:\n"
            "    print('RAISED', e)\n"
            "else:\n"
            "    print('OK' if ok else 'FAILED', getattr(g, 'last_error', None))\n")
    env = dict(os.environ, LFASM_LIBRARY=str(tmp_path / "absent.so"))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                         text=True, timeout=300).stdout
    assert "RAISED" in out and "no CPU fallback" in out, out
    import torch
    if not torch.cuda.is_available():
        env = {k: v for k, v in os.environ.items() if k != "LFASM_LIBRARY"}
        out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env,
                             capture_output=True, text=True, timeout=300).stdout
        assert "FAILED (2," in out, out
