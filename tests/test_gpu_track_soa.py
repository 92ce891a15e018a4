"""Tracks in SoA form at the boundary (gx_track_soa): the four stage calls
(gx_gpil, gx_propagate, gx_along_step, gx_post_step) against the oracle's
OneStep step by step, and the hand-over of live tracks between the engine and
the oracle (gx_transport_tracks).

With the FP64 parity variant the stage calls and the oracle take the same
operations in the same order, so after every step every track's state --
position, direction, energy, NIL, volume, stream, status -- and its
secondaries are the same bits on both sides."""
import numpy as np
import pytest
import torch
from oracle_ctypes import Tracks, oracle_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as g
    return g.ProxyDataManager()


def _compact(a, b):
    """Alive tracks of a, then alive tracks of b (TrackSoA), into a new SoA."""
    import geantexascalepilot_b200 as g
    ia = torch.nonzero(a.status[:a.n] == g.api.TRACK_ALIVE).flatten()
    ib = torch.nonzero(b.status[:b.n] == g.api.TRACK_ALIVE).flatten()
    out = g.TrackSoA(max(1, len(ia) + len(ib)))
    out.n = len(ia) + len(ib)
    for f in g.TrackSoA.INT_FIELDS + g.TrackSoA.DBL_FIELDS:
        getattr(out, f)[:out.n] = torch.cat([getattr(a, f)[ia], getattr(b, f)[ib]])
    ra, rb, ro = a.rng.view(6, a.capacity), b.rng.view(6, b.capacity), out.rng.view(6, out.capacity)
    ro[:, :out.n] = torch.cat([ra[:, ia], rb[:, ib]], 1)
    return out


def _compact_oracle(a, b):
    ia, ib = np.flatnonzero(a.status == 0), np.flatnonzero(b.status == 0)
    out = Tracks(len(ia) + len(ib))
    for f in ("type", "status", "event", "primary", "volume", "pos", "dir", "ekin", "nil", "msc", "rng"):
        getattr(out, f)[:] = np.concatenate([getattr(a, f)[ia], getattr(b, f)[ib]])
    return out


def _check_same(gpu, orc, what, step):
    """GPU TrackSoA.numpy() against oracle Tracks: status of every entry, full
    state of the alive ones."""
    st_g, st_o = gpu["status"], orc.status
    bad = np.flatnonzero(st_g != st_o)
    assert bad.size == 0, "%s, step %d: status differs at %s: gpu %s oracle %s" % (what, step, bad[:8], st_g[bad[:8]],
                                                                                   st_o[bad[:8]])
    alive = st_g == 0
    fields = {"type": (gpu["type"], orc.type), "volume": (gpu["volume"], orc.volume),
              "ekin": (gpu["ekin"], orc.ekin),
              "pos": (np.stack([gpu["x"], gpu["y"], gpu["z"]], 1), orc.pos),
              "dir": (np.stack([gpu["dx"], gpu["dy"], gpu["dz"]], 1), orc.dir),
              "nil": (np.stack([gpu["nil0"], gpu["nil1"], gpu["nil2"]], 1), orc.nil),
              "rng": (gpu["rng"].astype(np.float64), orc.rng)}
    for name, (a, b) in fields.items():
        a, b = a[alive], b[alive]
        diff = np.flatnonzero(np.any((a != b).reshape(len(a), -1), axis=1)) if len(a) else []
        assert len(diff) == 0, "%s, step %d: %s differs for alive track %d: gpu %r oracle %r" % (
            what, step, name, np.flatnonzero(alive)[diff[0]], a[diff[0]], b[diff[0]])


def _step_by_step(dm, oracle_gxm, cfg, prims, nvol, max_steps=100000):
    import geantexascalepilot_b200 as g
    cfg.precision, cfg.fp64_parity = 0, 1
    types, E, pos, d, _ = prims
    t = g.TrackSoA.from_primaries(cfg, types, E, pos, d)
    o = Tracks.from_soa(t.numpy())
    ocfg = oracle_config(cfg, 1)
    eg = torch.zeros((1, nvol), dtype=torch.float64, device="cuda")
    eo = np.zeros((1, nvol))
    steps_g = steps_o = 0
    for step in range(max_steps):
        if t.n == 0:
            break
        steps_g += int((t.status[:t.n] == 0).sum())
        g.gpil(dm, cfg, t)
        g.propagate(dm, cfg, t)
        g.along_step(dm, cfg, t, eg)
        sec = g.TrackSoA(2 * t.n)
        g.post_step(dm, cfg, t, sec, eg)
        osec, _, c = oracle_gxm.step_tracks(ocfg, o, eo)
        steps_o += c["steps"]
        _check_same(t.numpy(), o, "track", step)
        _check_same(sec.numpy(), osec, "secondary", step)
        t, o = _compact(t, sec), _compact_oracle(o, osec)
    assert t.n == 0
    assert steps_g == steps_o
    np.testing.assert_allclose(eg.cpu().numpy(), eo, rtol=1e-12, atol=1e-12 * eo.max())
    return steps_g, eo


def test_stages_match_the_oracle_step_by_step(dm, oracle_gxm):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(4)
    steps, eo = _step_by_step(dm, oracle_gxm, cfg, prims, nvol)
    ref = oracle_gxm.transport(oracle_config(cfg), *prims[:4], nvol=nvol)
    assert steps == ref["steps"]
    np.testing.assert_allclose(eo, ref["edep"], rtol=1e-12, atol=1e-12 * eo.max())


def test_stages_match_the_oracle_step_by_step_in_field(dm, oracle_gxm):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(2, 2)
    _step_by_step(dm, oracle_gxm, cfg, prims, nvol)


@pytest.mark.parametrize("engine", [0, 1])
def test_hand_over_to_the_oracle_continues_every_track(dm, oracle_gxm, engine):
    """k iterations on the GPU (FP64 parity variant), the tracks still alive
    handed to the oracle for the rest: steps and deposits add up to the
    oracle's own run of the same primaries."""
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(16)
    cfg.precision, cfg.engine, cfg.fp64_parity = 0, engine, 1
    types, E, pos, d, _ = prims
    t = g.TrackSoA.from_primaries(cfg, types, E, pos, d)
    out, eg, st = g.transport_tracks(dm, cfg, t, max_iterations=6, nvol=nvol)
    torch.cuda.synchronize()
    assert 0 < out.n < out.capacity
    rest = oracle_gxm.transport_tracks(oracle_config(cfg), Tracks.from_soa(out.numpy()), nvol)
    ref = oracle_gxm.transport(oracle_config(cfg), *prims[:4], nvol=nvol)
    assert st["steps"] + rest["steps"] == ref["steps"]
    total = eg.cpu().numpy() + rest["edep"]
    np.testing.assert_allclose(total, ref["edep"], rtol=1e-11, atol=1e-11 * ref["edep"].max())


@pytest.mark.parametrize("precision", [0, 1])
def test_hand_over_and_back_equals_one_run(dm, precision):
    """Stopped after 3 iterations and restarted from the tracks it wrote out,
    the batched engine gives what one uninterrupted run gives (FP32-mixed
    too: the float state goes out and back in exactly)."""
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(16, 16)
    cfg.precision, cfg.engine = precision, 1
    types, E, pos, d, _ = prims
    whole, st_w, _ = g.transport(dm, cfg, types, E, pos, d, nvol=nvol)
    t = g.TrackSoA.from_primaries(cfg, types, E, pos, d)
    out, e1, st1 = g.transport_tracks(dm, cfg, t, max_iterations=3, nvol=nvol)
    assert out.n > 0
    _, e2, st2 = g.transport_tracks(dm, cfg, out, max_iterations=0, nvol=nvol)
    torch.cuda.synchronize()
    assert st1["steps"] + st2["steps"] == st_w["steps"]
    w = whole.cpu().numpy()
    np.testing.assert_allclose(e1.cpu().numpy() + e2.cpu().numpy(), w, rtol=1e-9, atol=1e-9 * w.max())


def test_stage_calls_reject_what_they_do_not_offer(dm):
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import GxError, configs
    cfg, prims, nvol = configs.c2(2)
    t = g.TrackSoA.from_primaries(cfg, *prims[:4])
    cfg.msc = 1
    with pytest.raises(GxError, match="msc"):
        g.gpil(dm, cfg, t)
    cfg.msc = 0
    with pytest.raises(GxError, match="capacity 2 n"):
        g.post_step(dm, cfg, t, g.TrackSoA(1), torch.zeros((1, nvol), dtype=torch.float64, device="cuda"))
