"""The C-ABI library loads and exports every entry point include/gx_abi.h
declares (CPU only: no compute calls)."""
import ctypes
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "gx_abi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import geantexascalepilot_b200 as g
    lib = ctypes.CDLL(g.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(syms) == sorted(g.EXPORTED)


def test_version_and_error_string_without_gpu():
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200._lib import lib
    assert lib.gx_version() == 100
    assert isinstance(lib.gx_last_error_string(), bytes)
    # argument checks happen before any device call
    cfg = g.default_config()
    rc = lib.gx_transport_run(None, ctypes.byref(cfg), 0, None, None, None, None, None, None, 0, None, None, None)
    assert rc == -1 and b"null" in lib.gx_last_error_string()
