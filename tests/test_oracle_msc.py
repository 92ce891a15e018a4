"""Multiple scattering in the oracle (CPU): the restated Urban-type model's
first moment, its path-length conversion, the radiation lengths it uses, and
showers with it switched on.  The reference has no multiple-scattering model
(proxy/ProxyScattering.hpp is a placeholder), so the checks are the model's
defining properties; the GPU engine runs the same code path against this
oracle in test_gpu_transport.py."""
import numpy as np
import pytest


def test_radiation_lengths(oracle):
    # Tsai's formula (ProxyElementUtils.cu:40-61): lead 5.61 mm, liquid argon 140 mm
    assert abs(oracle.material(82.0, 207.2, 11.35)["radlen"] - 5.612) < 0.01
    assert abs(oracle.material(18.0, 39.95, 1.396)["radlen"] - 140.0) < 0.2


@pytest.mark.parametrize("Z,mat,E,t", [(82.0, 1, 1.0, 0.01), (82.0, 1, 10.0, 0.5), (82.0, 1, 0.2, 0.005),
                                       (82.0, 1, 1000.0, 50.0), (82.0, 1, 5.0, 2.0), (18.0, 2, 1.0, 0.05),
                                       (18.0, 2, 0.05, 0.001), (18.0, 2, 100.0, 3.0)])
def test_mean_cosine_is_exp_minus_tau(oracle, Z, mat, E, t):
    """<cos theta> = exp(-tau), tau = t / lambda1 averaged over a 2% loss."""
    X0 = oracle.material(Z, 207.2 if Z == 82 else 39.95, 11.35 if Z == 82 else 1.396)["radlen"]
    n = 200000
    st = oracle.substreams(np.full(6, 12345.0), 17, n)
    lam0, lam1 = oracle.msc_lambda1(1, mat, E), oracle.msc_lambda1(1, mat, 0.98 * E)
    c, _ = oracle.msc_cos(Z, X0, st, t, lam0, lam1, E, 0.98 * E)
    assert np.all((c >= -1.0) & (c <= 1.0))
    tau = t * np.log(lam0 / lam1) / (lam0 - lam1) if abs(lam1 - lam0) > 0.01 * lam0 else t / lam0
    assert abs(c.mean() - np.exp(-tau)) < 5 * c.std() / np.sqrt(n) + 1e-12


def test_central_width_follows_highland(oracle):
    """Small steps: the rms projected angle of the central part is of the
    order of the Highland width 13.6 MeV / (beta c p) sqrt(t / X0) (within
    the model's Z correction, +-20%)."""
    X0 = oracle.material(82.0, 207.2, 11.35)["radlen"]
    E, t = 50.0, 0.05
    lam = oracle.msc_lambda1(1, 1, E)
    st = oracle.substreams(np.full(6, 12345.0), 99, 100000)
    c, _ = oracle.msc_cos(82.0, X0, st, t, lam, lam, E, E)
    theta = np.arccos(np.clip(c, -1, 1))
    core = np.sort(theta)[: int(0.98 * len(theta))]
    me = 0.510998910
    bcp = E * (E + 2 * me) / (E + me)
    highland = 13.6 / bcp * np.sqrt(t / X0) * (1 + 0.038 * np.log(t / X0))
    assert 0.8 < np.sqrt(np.mean(core ** 2) / 2) / highland < 1.2


def test_path_length_conversion(oracle):
    for t, lam in ((0.3, 1.0), (1e-9, 1.0), (5.0, 0.1), (0.01, 50.0)):
        z, back = oracle.msc_paths(t, lam)
        assert z <= t
        np.testing.assert_allclose(z, lam * (1 - np.exp(-t / lam)) if t / lam > 1e-6 else t, rtol=1e-13)
        np.testing.assert_allclose(back, t, rtol=1e-9)


def test_showers_with_multiple_scattering(oracle):
    from oracle_ctypes import oracle_config
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(8)
    res = {}
    for msc in (0, 1, 2):
        c = oracle_config(cfg, 4)
        c.msc = msc
        res[msc] = r = oracle.transport(c, *prims[:4], nvol=nvol)
        e0 = prims[1].sum()
        assert r["errors"] == 0
        assert abs(r["edep"].sum() + r["escaped"] - e0) <= 1e-9 * e0
    # the extra step limit adds steps; the primaries' energy stays in the calorimeter
    assert res[1]["steps"] > 1.05 * res[0]["steps"]
    assert res[1]["edep"].sum() > 0.95 * prims[1].sum()
    # the lateral displacement moves tracks towards boundaries (smaller
    # safeties, so more safety-limited steps) without changing the shower's
    # scale
    assert res[1]["steps"] < res[2]["steps"] < 1.15 * res[1]["steps"]
    assert abs(res[2]["tracks"] - res[1]["tracks"]) < 0.03 * res[1]["tracks"]
    assert res[2]["edep"].sum() > 0.95 * prims[1].sum()
