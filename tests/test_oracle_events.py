"""Event generators on the CPU: the oracle's restatement of ProxyEgammaGun and
ProxyHepEvtGenerator against the reference's own output (tests/golden/
events.npz, from make_golden_events.py), and the library's host-side HEPEVT
reader against both, with the edge cases the reference leaves undefined."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SAMPLE = os.path.join(HERE, "golden", "hepevt_sample.data")


@pytest.fixture(scope="module")
def ev():
    return np.load(os.path.join(HERE, "golden", "events.npz"))


@pytest.mark.parametrize("name", ["gun_default", "gun_narrow"])
def test_oracle_gun_matches_reference_bit_for_bit(oracle, ev, name):
    ne, npart, gf, p0, p1, e0, e1, f0, f1 = ev[name + "_params"]
    pdg, p, ek, d, st = oracle.egamma_gun(ev[name + "_state"], int(ne), int(npart), gf, p0, p1, e0, e1, f0, f1)
    assert np.array_equal(pdg, ev[name + "_pdg"])
    assert np.array_equal(p, ev[name + "_p"])
    assert np.array_equal(ek, ev[name + "_ekin"])
    assert np.array_equal(d, ev[name + "_dir"])
    assert np.array_equal(st, ev[name + "_state_out"])


def test_oracle_gun_direction_setter_matches_reference(oracle, ev):
    for xyz, dref in zip(ev["dir_xyz"], ev["dir_ref"]):
        eta, phi = oracle.egamma_dir(0, *xyz)
        # the gun draws eta in [eta, eta]: an infinite eta (beam along z) gives
        # NaN there, in the reference too
        with np.errstate(invalid="ignore"):
            eta = eta + (eta - eta) * 0.5
        th = 2 * np.arctan(np.exp(-eta))
        d = np.array([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)])
        np.testing.assert_allclose(d, dref, rtol=0, atol=1e-15)


def test_package_direction_setter(oracle):
    import geantexascalepilot_b200 as gx
    for xyz in ([1.0, 0.5, 2.0], [0.3, -0.4, -5.0], [-1.0, 2.0, 0.5]):
        for mode in (gx.MODE_QUIRK, gx.MODE_PHYSICS):
            assert np.allclose(gx.set_direction_xyz(*xyz, mode=mode), oracle.egamma_dir(mode, *xyz), rtol=0,
                               atol=1e-15, equal_nan=True)
    # quirk mode: a beam along z gives an infinite eta, as in the reference
    assert gx.set_direction_xyz(0.0, 0.0, 1.0, mode=gx.MODE_QUIRK)[0] == np.inf
    # physics mode points along (x, y, z), also backwards and along the axis
    for xyz in ([0.3, -0.4, -5.0], [0.0, 0.0, 1.0], [0.0, 0.0, -2.0]):
        eta, phi = gx.set_direction_xyz(*xyz)
        eta = eta + (eta - eta) * 0.5
        th = 2 * np.arctan(np.exp(-eta))
        d = np.array([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)])
        np.testing.assert_allclose(d, np.array(xyz) / np.linalg.norm(xyz), atol=1e-15)


def test_hepevt_readers_match_reference(oracle, ev):
    import geantexascalepilot_b200 as gx
    o = oracle.hepevt(SAMPLE, 0)
    lib = gx.hepevt_read(SAMPLE, gx.MODE_QUIRK)
    for got in (o, lib):
        assert np.array_equal(got["event"], ev["hepevt_event"])
        assert np.array_equal(got["pdg"], ev["hepevt_pdg"])
        assert np.array_equal(got["ekin"], ev["hepevt_ekin"])
        assert np.array_equal(got["dir"], ev["hepevt_dir"])
        assert got["nevents"] == 12 and got["bad"] == 0
    assert np.array_equal(o["p"], ev["hepevt_p"])


def test_hepevt_physics_mode(oracle):
    import geantexascalepilot_b200 as gx
    q = gx.hepevt_read(SAMPLE, gx.MODE_QUIRK)
    ph = gx.hepevt_read(SAMPLE, gx.MODE_PHYSICS)
    o = oracle.hepevt(SAMPLE, 1)
    assert np.array_equal(ph["ekin"], o["ekin"]) and np.array_equal(ph["pdg"], q["pdg"])
    # massless photons: E = |p|, in MeV
    g = ph["pdg"] == 22
    np.testing.assert_allclose(ph["ekin"][g], 1000.0 * q["ekin"][g], rtol=1e-15)
    # massive: E = sqrt(p^2 + m^2) - m with the mass as given
    mass = {11: 0.510998910, -11: 0.510998910, 211: 139.57018, -211: 139.57018, 13: 105.6583745, -13: 105.6583745,
            2212: 938.272046}
    for code, m in mass.items():
        sel = ph["pdg"] == code
        if sel.any():
            pm = o["p"][sel]
            np.testing.assert_allclose(ph["ekin"][sel], np.sqrt(pm ** 2 + m ** 2) - m, rtol=1e-12)
    assert all(gx.pdg_to_type(c) == t for c, t in ((22, 0), (11, 1), (-11, 2), (211, -1), (13, -1)))


def test_hepevt_edge_cases(oracle, tmp_path):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import GxError
    empty = tmp_path / "empty.data"
    empty.write_text("")
    assert gx.hepevt_read(str(empty))["nevents"] == 0
    # a daughter range past the end of its event, and an event with no entries
    bad = tmp_path / "bad.data"
    bad.write_text("3\n2 23 2 5 0 0 1 91.2\n1 22 0 0 0 0 5 0\n1 11 0 0 0 1 0 0.000511\n0\n")
    r = gx.hepevt_read(str(bad))
    o = oracle.hepevt(str(bad), 1)
    assert r["nevents"] == o["nevents"] == 2 and r["bad"] == o["bad"] == 2
    assert list(r["pdg"]) == list(o["pdg"]) == [22, 11]
    trunc = tmp_path / "trunc.data"
    trunc.write_text("3\n2 23 2 3 0 0 1 91.2\n1 22 0 0 0 0 5 0\n")
    with pytest.raises(GxError):
        gx.hepevt_read(str(trunc))
    with pytest.raises(GxError):
        gx.hepevt_read(str(tmp_path / "missing.data"))
    # max_events stops early
    assert gx.hepevt_read(SAMPLE, max_events=3)["nevents"] == 3


SPOT_C4 = dict(types=(1, 2, 0), energy=(10.0, 1.0e5), cone_deg=5.0, axis=2, centre=(0.0, 0.0, -200.0),
               half=(10.0, 10.0))


def test_spot_gun_host_matches_oracle(oracle):
    """The library's host beam-spot gun (C4's generator) and the oracle's
    restatement: the same primaries from stream 1 of the seed, also when a
    shard starts at primary `first` (jumped, against drawn in sequence)."""
    import geantexascalepilot_b200 as gx
    seed = (12345.0,) * 6
    t, E, p, d = gx.spot_gun(3000, seed=seed, stream=1, device=False, **SPOT_C4)
    o = oracle.spot_gun(seed, 1, 0, 3000, SPOT_C4["types"], SPOT_C4["energy"], SPOT_C4["cone_deg"], SPOT_C4["axis"],
                        SPOT_C4["centre"], SPOT_C4["half"])
    for a, b in zip((t, E, p, d), o):
        np.testing.assert_array_equal(a, b)
    t2, E2, p2, d2 = gx.spot_gun(1000, seed=seed, stream=1, first=2000, device=False, **SPOT_C4)
    np.testing.assert_array_equal(E2, E[2000:])
    np.testing.assert_array_equal(d2, d[2000:])
    np.testing.assert_array_equal(t2, t[2000:])
    # C4's shape: types cycle, log-uniform energy, 5 degree cone, 2 x 2 cm spot
    assert list(t[:6]) == [1, 2, 0, 1, 2, 0]
    assert E.min() >= 10.0 and E.max() <= 1.0e5
    assert abs(np.log(E).mean() - 0.5 * (np.log(10.0) + np.log(1.0e5))) < 0.1
    assert np.all(d[:, 2] >= np.cos(np.radians(5.0)) - 1e-15)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, rtol=1e-15)
    assert np.all(np.abs(p[:, :2]) <= 10.0) and np.all(p[:, 2] == -200.0)
    # another stream, and the transport's substreams, are other numbers
    _, E0, _, _ = gx.spot_gun(10, seed=seed, stream=0, device=False, **SPOT_C4)
    assert not np.any(E0 == E[:10])


def test_spot_gun_rejects_bad_arguments():
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import GxError
    for bad in (dict(energy=(0.0, 1.0)), dict(energy=(2.0, 1.0)), dict(types=(3,)), dict(axis=3),
                dict(cone_deg=200.0), dict(stream=-1)):
        kw = dict(SPOT_C4)
        kw.update(bad)
        with pytest.raises(GxError):
            gx.spot_gun(4, device=False, **kw)
