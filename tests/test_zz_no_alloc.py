"""The allocation-free transport entry point, gx_transport_run_noalloc.

Some callers cannot call cudaMalloc while they run: a host framework whose
caching allocator already owns the device memory, a process held to a fixed
memory budget, or a time-critical loop that cannot take the device
synchronisation an allocation implies.  This entry point serves them from a
static device array inside the library; here it is called through the C ABI
and compared, on two calls in a row, with the allocating entry point
(gx_transport_run, plain FP64 loop) on the same inputs.  The file is named so
that pytest collects it last.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as g
    return g.ProxyDataManager()


def _device_prims(prims):
    types, E, pos, d, ev = prims
    return (torch.as_tensor(types, device="cuda"), torch.as_tensor(E, device="cuda"),
            torch.as_tensor(pos, device="cuda"), torch.as_tensor(d, device="cuda"),
            None if ev is None else torch.as_tensor(ev, device="cuda"))


@pytest.mark.parametrize("workload", ["c1", "c2"])
def test_noalloc_matches_allocating_entry_point_on_two_calls(dm, workload):
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c1(512) if workload == "c1" else configs.c2(2)
    cfg.precision, cfg.engine = 0, 0
    t, E, p, d, ev = _device_prims(prims)
    want, st_want, _ = g.transport(dm, cfg, t, E, p, d, events=ev, nvol=nvol)
    want = want.cpu().numpy()
    for call in range(2):
        edep = torch.zeros((cfg.nevents, nvol), dtype=torch.float64, device="cuda")
        got, st = g.transport_noalloc(dm, cfg, t, E, p, d, events=ev, nvol=nvol, edep=edep)
        torch.cuda.synchronize()
        got = got.cpu().numpy()
        assert st["errors"] == 0, call
        assert st["steps"] == st_want["steps"] and st["tracks"] == st_want["tracks"], call
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9 * want.max())


def test_noalloc_rejects_inputs_beyond_its_static_limit(dm):
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import GxError, configs
    cfg, prims, nvol = configs.c1(g.api.NOALLOC_MAX_PRIMARIES + 1)
    cfg.precision = 0
    t, E, p, d, ev = _device_prims(prims)
    with pytest.raises(GxError, match="static limit"):
        g.transport_noalloc(dm, cfg, t, E, p, d, nvol=nvol)
    cfg.precision = 1
    t, E, p, d, ev = _device_prims(configs.c1(4)[1])
    with pytest.raises(GxError, match="FP64 only"):
        g.transport_noalloc(dm, cfg, t, E, p, d, nvol=nvol)


def test_noalloc_accepts_exactly_its_primary_limit(dm):
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c1(g.api.NOALLOC_MAX_PRIMARIES)
    cfg.precision = 0
    t, E, p, d, ev = _device_prims(prims)
    got, st = g.transport_noalloc(dm, cfg, t, E, p, d, nvol=nvol)
    torch.cuda.synchronize()
    assert st["errors"] == 0 and st["tracks"] >= g.api.NOALLOC_MAX_PRIMARIES
    # with charged secondaries deposited locally (their kinetic energy), each
    # pair's two electron masses leave the ledger
    e_pairs = st["n_pair"] * 2 * 0.510998910
    assert abs(got.sum().item() + st["escaped"] + e_pairs - E.sum().item()) <= 1e-9 * E.sum().item()


def test_noalloc_overflow_returns_its_status_and_the_next_call_is_clean(dm):
    """More tracks in flight than the static array holds: 512 electrons of
    10 GeV injected at once (the injection throttle opened with a huge
    wave_energy) peak far above 16384 in flight plus 16384 deferred.  The call
    must end with GX_ERR_OVERFLOW, not hang, and score the tracks that did not
    fit; the next call, on the array this one left behind, must again equal
    the allocating entry point."""
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import GxError, configs
    from geantexascalepilot_b200._lib import GX_ERR_OVERFLOW
    cfg, prims, nvol = configs.c2(512)
    cfg.precision = 0
    prims = (prims[0], np.full(512, 1.0e4), prims[2], prims[3], prims[4])
    cfg.wave_energy = 1.0e12
    t, E, p, d, ev = _device_prims(prims)
    with pytest.raises(GxError, match="tracks in flight") as exc:
        g.transport_noalloc(dm, cfg, t, E, p, d, nvol=nvol)
    assert exc.value.code == GX_ERR_OVERFLOW
    torch.cuda.synchronize()
    cfg, prims, nvol = configs.c2(2)
    cfg.precision, cfg.engine = 0, 0
    t, E, p, d, ev = _device_prims(prims)
    want, st_want, _ = g.transport(dm, cfg, t, E, p, d, nvol=nvol)
    got, st = g.transport_noalloc(dm, cfg, t, E, p, d, nvol=nvol)
    torch.cuda.synchronize()
    assert st["errors"] == 0 and st["steps"] == st_want["steps"] and st["tracks"] == st_want["tracks"]
    np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-9, atol=1e-9 * want.max().item())
