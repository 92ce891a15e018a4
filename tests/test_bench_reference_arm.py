"""bench.py's reference arm (the CPU oracle on the C3 batch) builds its
workload without the CUDA library; here its primaries and oracle
configuration are checked against the package's C3 definition, and a small
run is checked to load no library of the package."""
import json
import os
import subprocess
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c3_definitions_match_the_package():
    sys.path.insert(0, REPO)
    import bench
    from geantexascalepilot_b200 import configs
    from oracle_ctypes import oracle_config
    cfg, prims, nvol = configs.c3(300, 200)
    mine = bench.c3_primaries(300, 200)
    for a, b in zip(mine, prims[:4]):
        assert np.array_equal(np.asarray(a), np.asarray(b)) and np.asarray(a).dtype == np.asarray(b).dtype
    want, got = oracle_config(cfg, 8), bench.c3_oracle_config(8)
    for name, _ in want._fields_:
        a, b = getattr(want, name), getattr(got, name)
        if hasattr(a, "__len__"):
            a, b = list(a), list(b)
        assert a == b, name
    assert nvol == 100


def test_reference_arm_loads_no_cuda_library():
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--electrons', '6', '--photons', '6',"
            " '--steps', '2', '--warmup', '1']; sys.path.insert(0, %r); import bench; bench.main();"
            " maps = open('/proc/self/maps').read();"
            " print('LOADED', any(m in sys.modules for m in ('geantexascalepilot_b200', 'torch')),"
            " 'libgxb200' in maps)" % REPO)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=REPO, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["ms_per_step"] > 0
    assert line["config"] == __import__("bench").c3_config_dict(6, 6)
    assert lines[1] == "LOADED False False"
