"""The C-ABI library loads and exports every function include/bbwadg.h
declares; argument validation needs no GPU.  CPU only."""
import ctypes
import os
import re

import pytest

from bbwadg_b200 import _lib

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "bbwadg.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bbw_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_status_strings():
    L = _lib.lib()
    assert L.bbw_status_string(0) == b"ok"
    assert L.bbw_status_string(7) == b"unsupported size or option"
    assert b"sm_100a" in L.bbw_version()


def test_argument_validation_without_gpu():
    L = _lib.lib()
    # invalid arguments are rejected before any CUDA call
    assert L.bbw_rk_volume(5, -1, None, None, None, None, None, None, None) == 1
    assert L.bbw_rk_surface(5, 10, 7, None, None, None, None, None, None, None) == 1
    assert L.bbw_rk_update(9, 10, 0.0, 0.0, 0.0, None, None, None, None) == 7
    assert L.bbw_create(None, None, 0, 0, None) == 1
    assert L.bbw_stage(None, 0.0, 0.0, 0.0) == 1
    assert b"NULL" in L.bbw_last_error() or L.bbw_last_error() != b""
    # K = 0 is a valid no-op, as an OCCA launch over an empty outer loop
    assert L.bbw_rk_volume(5, 0, None, None, None, None, None, None, None) == 0


def test_context_size_limits_without_gpu():
    """K and N outside the supported range are refused before any CUDA call:
    the neighbour code packs the element index above an 8-bit face
    permutation id, so K < 2^23."""
    import ctypes
    L = _lib.lib()
    h = ctypes.c_void_p()
    od = _lib.OpsDesc()
    for N, K, code in ((3, 1 << 23, 1), (3, 0, 1), (3, -5, 1), (0, 10, 7), (99, 10, 7)):
        md = _lib.MeshDesc(N=N, K=K, Nq=31)
        assert L.bbw_create(ctypes.byref(md), ctypes.byref(od), 0, 0, ctypes.byref(h)) == code
        assert not h.value
    md = _lib.MeshDesc(N=3, K=1 << 23, Nq=31)
    L.bbw_create(ctypes.byref(md), ctypes.byref(od), 0, 0, ctypes.byref(h))
    assert b"2^23" in L.bbw_last_error()


def test_kernel_level_node_index_limit_without_gpu():
    """Node indices are int32 (as the reference's vmapP): K * 4 * Np >= 2^31
    is refused before any CUDA call; the arrays are never touched."""
    L = _lib.lib()
    Np = 56  # N = 5
    K = (1 << 31) // (4 * Np) + 1
    assert L.bbw_rk_volume(5, K, 1, 1, 1, 1, 1, 1, None) == 7
    assert b"2^31" in L.bbw_last_error()
    assert L.bbw_rk_update(5, K, 0.0, 0.0, 0.0, 1, 1, 1, None) == 7
    assert L.bbw_rk_update_wadg(5, K, 95, 1, 1, 1, 1, 0.0, 0.0, 0.0, 1, 1, 1, None) == 7
