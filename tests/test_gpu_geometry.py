"""The CSG volume tree on the GPU: the device navigator against the oracle's
(same rays, same touchables), and transport through trees: the calorimeter
built as a tree against the layered navigator and against the oracle, a
geometry of rotated tubes, spheres and boxes in 4 T, both engines, FP32-mixed,
the field map."""
import numpy as np
import pytest
import torch

from oracle_ctypes import oracle_config
from test_csg import _rays, crowded_geometry, mixed_geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as g
    return g.ProxyDataManager()


def _run(dm, cfg, prims, nvol, **kw):
    import geantexascalepilot_b200 as gx
    for k, v in kw.items():
        setattr(cfg, k, v)
    edep, st, ps = gx.transport(dm, cfg, *prims[:4], events=prims[4], nvol=nvol, primary_steps=True)
    torch.cuda.synchronize()
    return edep.cpu().numpy(), st, ps.cpu().numpy()


@pytest.mark.parametrize("name", ["mixed", "crowded", "calorimeter"])
def test_probe_matches_oracle(dm, oracle, name):
    """locate, step, crossing and safety on 20000 rays: the same touchables
    and the same distances (products and sums are rounded separately on the
    device, as in the oracle; the device's slab grids over many children give
    the oracle's plain loops' results)"""
    from geantexascalepilot_b200 import geometry as G
    sigma = 80.0
    if name == "mixed":
        geo = mixed_geometry()
        centres = [(100, -50, 20), (-250, 150, 0), (0, 350, -100), (-300, -300, 300), (250, 200, -200),
                   (200, -250, 250), (-100, -350, -300), (350, -50, 350)]
    elif name == "crowded":
        geo = crowded_geometry()
        centres = [t["translation"] for t in geo.touchables() if t["parent"] >= 0]
        sigma = 20.0
    else:
        geo = G.calorimeter(axis=0)
        centres = [(-200.0 + 8.0 * k, 0.0, 0.0) for k in range(50)]
    geo.load(dm)
    h = oracle.csg_build(geo)
    p, d = _rays(20000, 3, centres, sigma)
    lim = np.where(np.arange(len(p)) % 4 == 0, 30.0, 1e30)
    ov, os_, on, osf = oracle.csg_probe(h, p, d, lim)
    gv, gs, gn, gsf = [t.cpu().numpy() for t in G.probe(dm, p, d, lim)]
    oracle.csg_free(h)
    assert np.array_equal(gv, ov)
    assert np.array_equal(gn, on)
    inside = ov >= 0
    assert inside.sum() > 8000
    assert (on != ov)[inside].sum() > 2000
    np.testing.assert_array_equal(gs[inside], os_[inside])
    np.testing.assert_array_equal(gsf[inside], osf[inside])


@pytest.mark.parametrize("precision", [0, 1])
def test_tree_calorimeter_equals_layered(dm, precision):
    from geantexascalepilot_b200 import configs, geometry as G
    cfg, prims, nvol = configs.c2(16)
    a, sa, pa = _run(dm, cfg, prims, nvol, precision=precision, engine=1)
    assert G.calorimeter(axis=cfg.axis).load(dm) == nvol
    b, sb, pb = _run(dm, cfg, prims, nvol, geometry=2)
    assert sb["errors"] == 0
    assert sa["steps"] == sb["steps"] and sa["tracks"] == sb["tracks"]
    assert np.array_equal(pa, pb)
    np.testing.assert_allclose(b, a, rtol=1e-9, atol=1e-9 * a.max())


def test_tree_calorimeter_matches_oracle(dm, oracle):
    from geantexascalepilot_b200 import configs, geometry as G
    cfg, prims, nvol = configs.c2(16)
    geo = G.calorimeter(axis=cfg.axis)
    geo.load(dm)
    g, st, _ = _run(dm, cfg, prims, nvol, precision=0, engine=1, geometry=2)
    h = oracle.csg_build(geo)
    oc = oracle_config(cfg)
    oc.csg = h
    ref = oracle.transport(oc, *prims[:4], nvol=nvol)
    oracle.csg_free(h)
    assert st["errors"] == 0
    assert abs(st["steps"] - ref["steps"]) <= 1e-5 * ref["steps"]
    np.testing.assert_allclose(g.ravel(), ref["edep"].ravel(), rtol=1e-6, atol=1e-6 * ref["edep"].max())


def _mixed_primaries(n):
    """e- and gamma at 2 GeV aimed at the solids of the mixed geometry"""
    rng = np.random.default_rng(17)
    targets = np.array([(100, -50, 20), (-250, 150, 0), (0, 350, -100), (-300, -300, 300)], float)
    start = np.array([0.0, 0.0, -550.0])
    tgt = targets[np.arange(n) % 4] + rng.normal(0, 10.0, (n, 3))
    d = tgt - start
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    types = np.where(np.arange(n) % 2 == 0, 1, 0).astype(np.int32)
    return types, np.full(n, 2000.0), np.tile(start, (n, 1)), d, None


def test_mixed_tree_in_field_matches_oracle(dm, oracle):
    """rotated tubes, spheres and boxes in 4 T: FP64 against the oracle
    (statistically: FMA rounding in the helix redirects a few tracks),
    energy conservation, and the plain engine against the batched one"""
    from geantexascalepilot_b200 import configs
    geo = mixed_geometry()
    nvol = geo.load(dm)
    cfg = configs.base_config(99)
    cfg.geometry, cfg.Bz = 2, 4.0
    prims = _mixed_primaries(64)
    g, st, _ = _run(dm, cfg, prims, nvol, precision=0, engine=1)
    e0 = prims[1].sum()
    assert st["errors"] == 0
    assert abs(g.sum() + st["escaped"] - e0) <= 1e-9 * e0
    assert g.sum() > 0.3 * e0
    h = oracle.csg_build(geo)
    oc = oracle_config(cfg)
    oc.csg = h
    ref = oracle.transport(oc, *prims[:4], nvol=nvol)
    oracle.csg_free(h)
    assert abs(st["steps"] - ref["steps"]) <= 0.03 * ref["steps"]
    o = ref["edep"].ravel()
    big = o > 0.01 * o.sum()
    assert np.all(np.abs(g.ravel() - o)[big] <= 0.15 * o[big] + 2e-3 * o.sum())
    p, sp, _ = _run(dm, cfg, prims, nvol, precision=0, engine=0)
    assert sp["steps"] == st["steps"] and sp["tracks"] == st["tracks"]
    np.testing.assert_allclose(p, g, rtol=1e-9, atol=1e-9 * g.max())
    f, sf, _ = _run(dm, cfg, prims, nvol, precision=1, engine=1)
    cfg.engine = 1
    assert sf["errors"] == 0 and abs(f.sum() + sf["escaped"] - e0) <= 1e-5 * e0
    assert abs(sf["steps"] - st["steps"]) <= 0.03 * st["steps"]


def test_tree_with_field_map(dm):
    """the CMS map through the tree calorimeter (both kernel variant bits)"""
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs, geometry as G
    d = gx.ProxyDataManager()
    d.load_field_map()
    cfg, prims, nvol = configs.c3(12, 12)
    G.calorimeter(axis=cfg.axis).load(d)
    a, sa, _ = _run(d, cfg, prims, nvol, precision=1, engine=1, field_map=1, geometry=1)
    b, sb, _ = _run(d, cfg, prims, nvol, geometry=2)
    d.close()
    e0 = prims[1].sum()
    for e, s in ((a, sa), (b, sb)):
        assert s["errors"] == 0 and abs(e.sum() + s["escaped"] - e0) <= 1e-5 * e0
    assert abs(sa["steps"] - sb["steps"]) <= 0.02 * sa["steps"]
    la, lb = a.reshape(-1, 2).sum(1), b.reshape(-1, 2).sum(1)
    big = la > 0.002 * la.sum()
    assert np.all(np.abs(la - lb)[big] <= 5 * 0.2 / np.sqrt(24) * la[big] + 1e-3 * la.sum())


def test_geometry_errors(dm):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs, geometry as G
    cfg, prims, nvol = configs.c2(2)
    cfg.geometry = 2
    G.calorimeter(axis=cfg.axis).load(dm)
    with pytest.raises(gx.GxError, match="scored touchables"):
        gx.transport(dm, cfg, *prims[:4], nvol=nvol + 1)
    d2 = gx.ProxyDataManager()
    with pytest.raises(gx.GxError, match="volume tree"):
        gx.transport(d2, cfg, *prims[:4], nvol=nvol)
    d2.close()
