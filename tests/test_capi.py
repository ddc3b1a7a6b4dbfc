"""The C-ABI library loads and exports every function include/rtpg.h declares (no GPU)."""
import ctypes

from rtlib_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) > 20
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_signatures_cover_header():
    declared = set(_lib.declared_symbols())
    assert declared == set(_lib._SIGS), sorted(declared ^ set(_lib._SIGS))


def test_version_and_limits():
    L = _lib.lib()
    assert L.rtpg_version() >= 100
    a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    assert L.rtpg_query_limits(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) == 0
    assert a.value == 16384 and b.value == 31 and c.value == 32


def test_errors_without_device():
    """Bad arguments are rejected on the host with a message, before any CUDA call."""
    L = _lib.lib()
    assert L.rtpg_sdtree_destroy(None) == -1
    assert b"null" in L.rtpg_last_error()
    assert L.rtpg_sdtree_create(None, None, 20, 0.3, None, None) == -1
