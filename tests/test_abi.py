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
