"""Event generators on the GPU, through the C ABI: the device particle gun
against the reference's ProxyEgammaGun output (golden) and the oracle at
sizes where threads start mid-stream; HEPEVT primaries loaded into device
arrays; a transport fed straight from the gun."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
SAMPLE = os.path.join(HERE, "golden", "hepevt_sample.data")


@pytest.fixture(scope="module")
def ev():
    return np.load(os.path.join(HERE, "golden", "events.npz"))


def _gun(name, ev, **kw):
    import geantexascalepilot_b200 as gx
    ne, npart, gf, p0, p1, e0, e1, f0, f1 = ev[name + "_params"]
    out = gx.egamma_gun(int(ne), int(npart), gamma_fraction=gf, momentum=(p0, p1), eta=(e0, e1), phi=(f0, f1),
                        seed=tuple(ev[name + "_state"]), **kw)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("name", ["gun_default", "gun_narrow"])
def test_gun_matches_reference(ev, name):
    t, E, pos, d, evt, pdg = _gun(name, ev, vertex=(1.0, -2.0, 3.0))
    assert np.array_equal(pdg, ev[name + "_pdg"])
    assert np.array_equal(t, np.where(ev[name + "_pdg"] == 22, 0, 1))
    # momentum and kinetic energy: the same operations, no contraction -> exact
    assert np.array_equal(E, ev[name + "_ekin"])
    # direction: CUDA's sin / cos / atan / exp against glibc's, a few ulp
    np.testing.assert_allclose(d, ev[name + "_dir"], rtol=0, atol=1e-15)
    ne, npart = int(ev[name + "_params"][0]), int(ev[name + "_params"][1])
    assert np.array_equal(evt, np.repeat(np.arange(ne), npart))
    assert np.all(pos == np.array([1.0, -2.0, 3.0]))


def test_gun_long_stream_and_continuation(oracle):
    """300k particles (threads start deep in the stream by skip-ahead) against
    the oracle's sequential draws, and a second call continuing the stream."""
    import geantexascalepilot_b200 as gx
    seed = (12345.0,) * 6
    ne, npart = 3000, 100
    t, E, pos, d, evt, pdg = [o.cpu().numpy() for o in gx.egamma_gun(ne, npart, momentum=(10.0, 1.0e4), seed=seed)]
    opdg, _, oek, od, st = oracle.egamma_gun(np.array(seed), ne, npart, 0.5, 10.0, 1.0e4, -3.0, 3.0, 0.0,
                                             2 * np.pi)
    assert np.array_equal(pdg, opdg) and np.array_equal(E, oek)
    np.testing.assert_allclose(d, od, rtol=0, atol=1e-15)
    # the next 5 events from where the first call stopped
    t2, E2, _, _, ev2, pdg2 = [o.cpu().numpy() for o in gx.egamma_gun(5, npart, momentum=(10.0, 1.0e4), seed=seed,
                                                                       first_draw=4 * ne * npart, first_event=ne)]
    opdg2, _, oek2, _, _ = oracle.egamma_gun(st, 5, npart, 0.5, 10.0, 1.0e4, -3.0, 3.0, 0.0, 2 * np.pi)
    assert np.array_equal(pdg2, opdg2) and np.array_equal(E2, oek2)
    assert ev2.min() == ne and ev2.max() == ne + 4


def test_gun_rejects_bad_arguments():
    import geantexascalepilot_b200 as gx
    with pytest.raises(gx.GxError):
        gx.egamma_gun(2, 2, momentum=(10.0, 1.0))
    with pytest.raises(gx.GxError):
        gx.egamma_gun(2, 2, seed=(1.5, 1, 1, 1, 1, 1))
    assert gx.egamma_gun(0, 5)[0].numel() == 0


def test_hepevt_load_to_device():
    import geantexascalepilot_b200 as gx
    host = gx.hepevt_read(SAMPLE, gx.MODE_PHYSICS)
    (t, E, pos, d, evt), (nev, skipped) = gx.hepevt_load(SAMPLE, gx.MODE_PHYSICS, vertex=(0.0, 0.0, -150.0))
    keep = np.array([gx.pdg_to_type(c) >= 0 for c in host["pdg"]])
    assert nev == 12 and skipped == int((~keep).sum()) and t.numel() == int(keep.sum())
    assert np.array_equal(t.cpu().numpy(), [gx.pdg_to_type(c) for c in host["pdg"][keep]])
    assert np.array_equal(E.cpu().numpy(), host["ekin"][keep])
    assert np.array_equal(d.cpu().numpy(), host["dir"][keep])
    assert np.array_equal(evt.cpu().numpy(), host["event"][keep])
    assert torch.all(pos[:, 2] == -150.0)


def test_transport_from_the_gun():
    """Gun primaries go straight into the transport (no host copy): C2
    calorimeter, 100-500 MeV e-/gamma from the front face along +z."""
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs
    dm = gx.ProxyDataManager()
    cfg, _, nvol = configs.c2(1)
    cfg.nevents = 8
    eta, phi = gx.set_direction_xyz(0.0, 0.0, 1.0)
    t, E, pos, d, evt, pdg = gx.egamma_gun(8, 32, momentum=(100.0, 500.0), eta=(eta, eta), phi=(phi, phi),
                                           vertex=(0.0, 0.0, -200.0))
    edep, st, _ = gx.transport(dm, cfg, t, E, pos, d, events=evt, nvol=nvol)
    torch.cuda.synchronize()
    assert st["errors"] == 0 and st["steps"] > 256
    e0 = E.sum().item()
    assert abs(edep.sum().item() + st["escaped"] - e0) <= 1e-9 * e0
    assert edep.shape == (8, nvol) and torch.all(edep.sum(1) > 0)
    dm.close()


def test_spot_gun_device_equals_host():
    """the device beam-spot gun (each thread jumps to its first draw) writes
    the host version's primaries: positions and types exactly, energies and
    directions to the last bits of the device's exp / log / sin / cos"""
    import geantexascalepilot_b200 as gx
    kw = dict(types=(1, 2, 0), energy=(10.0, 1.0e5), cone_deg=5.0, axis=0, centre=(-200.0, 1.0, 2.0),
              half=(10.0, 5.0), seed=(7.0,) * 6, stream=1)
    for first, n in ((0, 50000), (12345, 777)):
        h = gx.spot_gun(n, first=first, device=False, **kw)
        g = [x.cpu().numpy() for x in gx.spot_gun(n, first=first, device=True, **kw)]
        np.testing.assert_array_equal(g[0], h[0])
        np.testing.assert_array_equal(g[2], h[2])
        np.testing.assert_allclose(g[1], h[1], rtol=1e-14)
        np.testing.assert_allclose(g[3], h[3], rtol=1e-14, atol=1e-15)
