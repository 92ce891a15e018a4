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
