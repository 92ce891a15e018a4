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


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the ABI's structures have the C compiler's size
    and field offsets (a config struct shorter than the library's would be
    overrun by gx_transport_config_default)."""
    import subprocess
    from geantexascalepilot_b200 import _lib as L
    pairs = {"gx_model_params": L.ModelParams, "gx_transport_config": L.TransportConfig,
             "gx_transport_stats": L.TransportStats, "gx_egamma_gun_params": L.GunParams,
             "gx_spot_gun_params": L.SpotGunParams, "gx_track_soa": L.TrackSoAStruct,
             "gx_autotune_report": L.AutotuneReport}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gx_abi.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)])
    got = dict(l.split() for l in subprocess.check_output([str(exe)], text=True).splitlines())
    for cname, py in pairs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert int(got["%s.%s" % (cname, f[0])]) == getattr(py, f[0]).offset, (cname, f[0])
