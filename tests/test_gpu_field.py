"""The field map on the GPU: the device lookup against the reference's reader
(golden), Runge-Kutta transport through a uniform map against the helix,
through the CMS map against the oracle, and energy conservation."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as gx
    d = gx.ProxyDataManager()
    d.load_field_map()
    return d


def test_device_lookup_matches_reference(dm):
    z = np.load(os.path.join(HERE, "golden", "field.npz"))
    B = dm.field_value(z["pos"]).cpu().numpy()
    np.testing.assert_allclose(B, z["B"], rtol=1e-13, atol=1e-15)


def _uniform_map(path, bz):
    with open(path, "w") as f:
        for ir in range(181):
            for iz in range(161):
                f.write("R(mm)= %g phi(deg)= 0 Z(mm)= %g   Bz(tesla)= %.9g Br(tesla)= 0 Bphi(tesla)= 0\n"
                        % (50.0 * ir, -16000.0 + 200.0 * iz, bz))


def _run(dm, cfg, prims, nvol, **kw):
    import geantexascalepilot_b200 as gx
    for k, v in kw.items():
        setattr(cfg, k, v)
    edep, st, _ = gx.transport(dm, cfg, *prims[:4], events=prims[4], nvol=nvol)
    torch.cuda.synchronize()
    return edep.cpu().numpy(), st


def test_runge_kutta_in_uniform_map_agrees_with_helix(tmp_path):
    """A map of 4 T along z everywhere: the Runge-Kutta sub-steps and the exact
    helix transport the same showers within statistics (C3 geometry, FP64)."""
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs
    path = str(tmp_path / "uniform.txt")
    _uniform_map(path, 4.0)
    d = gx.ProxyDataManager()
    d.load_field_map(path)
    B = d.field_value([[0.0, 0.0, 0.0], [123.0, -45.0, 6.0]]).cpu().numpy()
    np.testing.assert_allclose(B, [[0, 0, 4.0], [0, 0, 4.0]], rtol=1e-6, atol=1e-12)
    cfg, prims, nvol = configs.c3(24, 24)
    cfg.precision, cfg.engine = 0, 1
    a, sa = _run(d, cfg, prims, nvol, field_map=0)
    b, sb = _run(d, cfg, prims, nvol, field_map=1)
    d.close()
    for e, st in ((a, sa), (b, sb)):
        assert st["errors"] == 0 and abs(e.sum() + st["escaped"] - prims[1].sum()) <= 1e-9 * prims[1].sum()
    la, lb = a.reshape(-1, 2).sum(1), b.reshape(-1, 2).sum(1)
    big = la > 0.002 * la.sum()
    assert np.all(np.abs(la - lb)[big] <= 5 * 0.2 / np.sqrt(48) * la[big] + 1e-3 * la.sum())
    assert abs(sa["steps"] - sb["steps"]) <= 0.02 * sa["steps"]


def test_cms_map_fp64_matches_oracle(dm, oracle):
    """Through the CMS map (about 3.8 T at the calorimeter): the FP64 engine
    and the oracle run the same Runge-Kutta sub-steps on the same streams;
    rounding differences (FMA) redirect a few tracks, so compare statistically."""
    from oracle_ctypes import oracle_config
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(16, 16)
    cfg.precision, cfg.engine = 0, 1
    g, st = _run(dm, cfg, prims, nvol, field_map=1)
    cfg.field_map = 0
    c = oracle_config(cfg)
    h = oracle.field_map_load(os.path.join(os.path.dirname(HERE), "geantexascalepilot_b200", "data", "field",
                                           "cmsmagfield2015.txt"))
    c.field_map = h
    ref = oracle.transport(c, *prims[:4], nvol=nvol)
    assert st["errors"] == 0 and ref["errors"] == 0
    assert abs(st["steps"] - ref["steps"]) <= 0.01 * ref["steps"]
    e0 = prims[1].sum()
    assert abs(g.sum() + st["escaped"] - e0) <= 1e-9 * e0
    lg, lo = g.reshape(-1, 2).sum(1), ref["edep"].reshape(-1, 2).sum(1)
    big = lo > 0.002 * lo.sum()
    assert np.all(np.abs(lg - lo)[big] <= 5 * 0.2 / np.sqrt(32) * lo[big] + 1e-3 * lo.sum())


def test_cms_map_fp32_mixed_and_missing_map(dm):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(8, 8)
    cfg.precision, cfg.engine = 1, 1
    e, st = _run(dm, cfg, prims, nvol, field_map=1, msc=1)
    cfg.field_map = cfg.msc = 0
    assert st["errors"] == 0 and abs(e.sum() + st["escaped"] - prims[1].sum()) <= 1e-5 * prims[1].sum()
    bare = gx.ProxyDataManager()
    with pytest.raises(gx.GxError):
        _run(bare, cfg, prims, nvol, field_map=1)
    cfg.field_map = 0
    bare.close()
