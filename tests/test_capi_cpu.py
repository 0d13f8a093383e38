"""CPU checks of the C ABI: the library loads and exports every declared entry point."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "tdp1375.h")).read()
    return sorted(set(re.findall(r"\b(tdp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native_lib):
    names = declared_symbols()
    assert "tdp_search" in names and "tdp_pi_filter" in names
    for name in names:
        assert hasattr(native_lib, name), name


def test_binding_covers_header():
    from tdp1375_b200 import native
    assert sorted(native.SIGNATURES) == declared_symbols()


def test_struct_layouts():
    from tdp1375_b200 import native
    assert ctypes.sizeof(native.Instance) == 136
    assert ctypes.sizeof(native.Result) == 208
    assert ctypes.sizeof(native.Stats) == 8 * 8 + 8 + 8 + 5 * 8
    assert ctypes.sizeof(native.EngineConfig) == 48


def test_errors_without_slots(native_lib):
    """Calls on a slot that does not exist fail with the reference's message."""
    from tdp1375_b200 import native
    native_lib.tdp_destroy_slots()
    depth = ctypes.c_int32()
    out = (ctypes.c_int32 * 45)()
    buf = (ctypes.c_uint8 * 4)(0, 1, 2, 3)
    rc = native_lib.tdp_search(0, buf, buf, 4, 4, ctypes.c_float(1.45), 3, 0, out, ctypes.byref(depth))
    assert rc == native.ERR_SLOT and native.last_error() == "invalid slot"
    rc = native_lib.tdp_search(0, buf, buf, 64, 4, ctypes.c_float(1.45), 3, 0, out, ctypes.byref(depth))
    assert rc == native.ERR_ARGUMENT and "MAX_N" in native.last_error()
    rc = native_lib.tdp_search(0, buf, buf, 4, 4, ctypes.c_float(1.45), 16, 0, out, ctypes.byref(depth))
    assert rc == native.ERR_ARGUMENT and "maximumDepth" in native.last_error()


def test_pi_filter_argument_errors(native_lib):
    from tdp1375_b200 import native
    cyc = (ctypes.c_uint8 * 3)(0, 1, 9)
    tri = (ctypes.c_uint8 * 3)(0, 1, 2)
    out = (ctypes.c_uint8 * 8)()
    assert native_lib.tdp_pi_filter(cyc, 3, tri, 3, 64, 0, out, 1) == native.ERR_ARGUMENT
    assert native_lib.tdp_pi_filter(cyc, 3, tri, 3, 5, 0, out, 1) == native.ERR_ARGUMENT
    assert "out of range" in native.last_error()


def test_canonical_rejects_bad_rows(native_lib):
    """Rows are validated on the host before any device work."""
    import numpy as np
    from tdp1375_b200 import native
    vp = ctypes.c_void_p
    spi = np.zeros((1, 64), np.uint8)
    spi[0, :4] = [1, 0, 2, 3]  # fixed points 2 and 3
    ns = np.array([4], np.uint8)
    sig = np.zeros((1, 64), np.float32)
    h = np.zeros(1, np.int32)
    v = np.zeros(1, np.int32)
    rc = native_lib.tdp_canonical(spi.ctypes.data_as(vp), ns.ctypes.data_as(vp), 1, sig.ctypes.data_as(vp),
                                  h.ctypes.data_as(vp), v.ctypes.data_as(vp))
    assert rc == native.ERR_ARGUMENT and "fixed points" in native.last_error()
    ns[0] = 64
    rc = native_lib.tdp_canonical(spi.ctypes.data_as(vp), ns.ctypes.data_as(vp), 1, sig.ctypes.data_as(vp),
                                  h.ctypes.data_as(vp), v.ctypes.data_as(vp))
    assert rc == native.ERR_ARGUMENT and "2..63" in native.last_error()
