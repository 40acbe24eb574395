"""The C-ABI library loads and exports every entry point include/hops_b200.h
declares (no GPU needed: nothing here launches a kernel)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hops_b200.h")
LIB = os.path.join(ROOT, "mesohops_b200", "lib", "libhops_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(hops_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("hops_rk4_propagate", "hops_dsystem_dt", "hops_resident_propagate",
              "hops_noise_filter", "hops_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        from mesohops_b200.build import build
        build()
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls():
    from mesohops_b200 import _lib
    L = _lib.lib()
    assert L.hops_version() >= 10000
    assert L.hops_scalar_workspace_doubles(2, 2, 2, 3) > 0
    assert L.hops_resident_scalar_doubles(2, 2, 2) > 0
    assert L.hops_noise_filter_work_doubles(2, 10) >= 4 * 2 * 18
    # argument validation happens before any CUDA call
    rc = L.hops_resident_propagate(None, 0, 0, 0, 0, 1, None)
    assert rc == _lib.HOPS_EINVAL
    assert b"bad resident" in L.hops_last_error()


def test_noise_entry_points_validate_before_any_cuda_call():
    from mesohops_b200 import _lib
    L = _lib.lib()
    # no seed states, no rows, unknown sampler
    assert L.hops_noise_draw(None, 1, None, 1, 10, 0, None, None) == _lib.HOPS_EINVAL
    assert b"hops_noise_draw" in L.hops_last_error()
    assert L.hops_noise_draw(8, 1, 8, 1, 10, 7, 8, None) == _lib.HOPS_EINVAL
    assert L.hops_noise_draw(8, 1, 8, 1, 1, 0, 8, None) == _lib.HOPS_EINVAL
    # rows that are not a multiple of the shared correlation functions
    rc = L.hops_noise_filter_shared(8, 3, 8, 10, 20, 8, None, 8, None, None)
    assert rc == _lib.HOPS_EINVAL
    assert b"n_alpha=3 n_rows=10" in L.hops_last_error()
