"""Production-cut conversion on the CPU: the oracle's restatement and the
library's (host code) against the reference's own converter (golden
tests/golden/cuts.npz, make_golden_cuts.py), and against the cut table the
reference ships (cut.dat, written by Geant4 for a 0.7 mm cut)."""
import ctypes as C
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "cuts.npz"))


def _oracle_convert(oracle, p, Z, n, rho, cut, from_length):
    f = oracle.lib.gxo_cut_convert
    f.restype = C.c_double
    f.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double, C.c_int]
    return f(p, len(Z), (C.c_double * len(Z))(*Z), (C.c_double * len(n))(*n), rho, cut, from_length)


def test_converters_match_reference(oracle, golden):
    import geantexascalepilot_b200 as gx
    for name in golden["names"]:
        Z, n, rho = list(golden[name + "_Z"]), list(golden[name + "_n"]), float(golden[name + "_rho"])
        for p in range(3):
            for k, c in enumerate(golden["cuts_mm"]):
                ref = golden[name + "_energy"][p, k]
                assert _oracle_convert(oracle, p, Z, n, rho, c, 1) == pytest.approx(ref, rel=1e-13)
                assert gx.cut_convert(p, Z, n, rho, c) == pytest.approx(ref, rel=1e-13)
            for k, c in enumerate(golden["cuts_mev"]):
                ref = golden[name + "_length"][p, k]
                assert _oracle_convert(oracle, p, Z, n, rho, c, 0) == pytest.approx(ref, rel=1e-13)
                assert gx.cut_convert(p, Z, n, rho, c, from_length=False) == pytest.approx(ref, rel=1e-13)


def test_shipped_cut_table_is_reproduced(golden):
    """cut.dat (Geant4, 0.7 mm): e-/e+ to 1e-6, gamma within the converter's
    own 1% bisection tolerance."""
    t = open(os.path.join(os.path.dirname(HERE), "geantexascalepilot_b200", "data", "table", "cut.dat")).read().split()
    kev = np.array(t[2:2 + 24], dtype=float).reshape(12, 2)[:, 1].reshape(4, 3)
    k07 = list(golden["cuts_mm"]).index(0.7)
    for m, name in enumerate(["Galactic", "Pb", "LAr"]):
        mine = golden[name + "_energy"][:, k07] * 1e3
        np.testing.assert_allclose(mine[1:], kev[1:3, m], rtol=1e-6)
        assert abs(mine[0] / kev[0, m] - 1) < 0.01


def test_bad_arguments():
    import geantexascalepilot_b200 as gx
    with pytest.raises(gx.GxError):
        gx.cut_convert(3, 82, 3e19, 11.35, 0.7)
    with pytest.raises(gx.GxError):
        gx.cut_convert(1, 82, 3e19, 11.35, -1.0)
    with pytest.raises(gx.GxError):
        gx.cut_convert(1, 0.5, 3e19, 11.35, 0.7)
