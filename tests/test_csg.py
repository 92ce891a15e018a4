"""The CSG volume tree (transport geometry 2) on the CPU: the oracle's
navigator against direct geometric checks (point-in-solid by definition,
sampled along rays and over safety spheres), the oracle's step loop on the
tree-built calorimeter against its layered navigator, and the library's host
builder (gx_geom_*) against the oracle's flattening."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle_ctypes import oracle_config


def hex_prism(apothem, half_z):
    """a hexagonal prism as a convex polyhedron (8 planes)"""
    from geantexascalepilot_b200 import geometry as G
    planes = [[math.cos(k * math.pi / 3), math.sin(k * math.pi / 3), 0.0, apothem] for k in range(6)]
    return G.ConvexPolyhedron(planes + [[0, 0, 2.0, 2.0 * half_z], [0, 0, -1.0, half_z]])


def mixed_geometry():
    """boxes, tubes, spheres, trapezoids and a hexagonal prism, rotated and
    nested, in a Galactic world"""
    from geantexascalepilot_b200 import geometry as G
    world = G.LogicalVolume("world", G.UnplacedBox(600.0, 600.0, 600.0))
    tube = G.LogicalVolume("tube", G.UnplacedTube(50.0, 150.0, 100.0))
    tube.SetMaterialPtr("G4_Pb")
    tube.SetScored()
    shell = G.LogicalVolume("shell", G.UnplacedSphere(20.0, 60.0))
    shell.SetMaterialPtr("G4_lAr")
    shell.SetScored()
    box = G.LogicalVolume("box", G.UnplacedBox(30.0, 40.0, 50.0))
    box.SetMaterialPtr("G4_Pb")
    box.SetScored()
    orb = G.LogicalVolume("orb", G.UnplacedOrb(10.0))
    orb.SetMaterialPtr("G4_lAr")
    orb.SetScored()
    rod = G.LogicalVolume("rod", G.UnplacedTube(0.0, 8.0, 30.0))
    rod.SetMaterialPtr("G4_lAr")
    rod.SetScored()
    wedge = G.LogicalVolume("wedge", G.UnplacedTrd(3.0, 8.0, 4.0, 6.0, 7.0))
    wedge.SetMaterialPtr("G4_Pb")
    wedge.SetScored()
    trd = G.LogicalVolume("trd", G.UnplacedTrd("trd", 20.0, 40.0, 15.0, 30.0, 25.0))
    trd.SetMaterialPtr("G4_Pb")
    trd.SetScored()
    hexa = G.LogicalVolume("hex", hex_prism(30.0, 40.0))
    hexa.SetMaterialPtr("G4_lAr")
    hexa.SetScored()
    box.PlaceDaughter("orb", orb, G.Transformation3D(5.0, -10.0, 20.0))
    box.PlaceDaughter("rod", rod, G.Transformation3D(-12.0, 15.0, -10.0, 0.0, 90.0, 0.0))
    box.PlaceDaughter("wedge", wedge, G.Transformation3D(15.0, 20.0, -30.0, 10.0, 0.0, 0.0))
    arc = G.LogicalVolume("arc", G.UnplacedTube(40.0, 90.0, 60.0, 0.3, math.radians(100.0)))
    arc.SetMaterialPtr("G4_Pb")
    arc.SetScored()
    horseshoe = G.LogicalVolume("horseshoe", G.UnplacedTube("hs", 0.0, 70.0, 50.0, -1.0, math.radians(270.0)))
    horseshoe.SetMaterialPtr("G4_lAr")
    horseshoe.SetScored()
    world.PlaceDaughter("arc", arc, G.Transformation3D(-100.0, -350.0, -300.0, 10.0, 60.0, 0.0))
    world.PlaceDaughter("horseshoe", horseshoe, G.Transformation3D(350.0, -50.0, 350.0))
    world.PlaceDaughter("trd", trd, G.Transformation3D(250.0, 200.0, -200.0, 20.0, 30.0, 40.0))
    world.PlaceDaughter("hex", hexa, G.Transformation3D(200.0, -250.0, 250.0, 0.0, 35.0, 10.0))
    world.PlaceDaughter("tube", tube, G.Transformation3D(100.0, -50.0, 20.0, 30.0, 40.0, 0.0))
    world.PlaceDaughter("shell", shell, G.Transformation3D(-250.0, 150.0, 0.0))
    world.PlaceDaughter("box_a", box, G.Transformation3D(0.0, 350.0, -100.0, 0.0, 90.0, 45.0))
    world.PlaceDaughter("box_b", box, G.Transformation3D(-300.0, -300.0, 300.0, 10.0, 20.0, 30.0))
    gm = G.GeoManager()
    gm.SetWorld(world.Place())
    return gm.CloseGeometry()


def crowded_geometry():
    """a world holding 40 rotated boxes, tubes and spheres (its children get
    the slab grid), one of them holding 12 more"""
    from geantexascalepilot_b200 import geometry as G
    rng = np.random.default_rng(23)
    world = G.LogicalVolume("world", G.UnplacedBox(800.0, 800.0, 800.0))
    holder = G.LogicalVolume("holder", G.UnplacedBox(60.0, 60.0, 60.0))
    holder.SetMaterialPtr("G4_lAr")
    holder.SetScored()
    for k in range(12):
        pin = G.LogicalVolume("pin%d" % k, G.UnplacedTube(0.0, 3.0, 50.0))
        pin.SetMaterialPtr("G4_Pb")
        pin.SetScored()
        holder.PlaceDaughter("pin%d" % k, pin, G.Transformation3D(-44.0 + 8.0 * k, 0.0, 0.0))
    for k in range(40):
        x, y, z = -650.0 + 32.0 * k, rng.uniform(-600, 600), rng.uniform(-600, 600)
        if k == 20:
            world.PlaceDaughter("holder", holder, G.Transformation3D(x, y, z, 15.0, 25.0, 35.0))
            continue
        kind = k % 4
        solid = (G.UnplacedBox(12.0, 40.0, 30.0) if kind == 0 else
                 G.UnplacedTube(4.0, 14.0, 40.0) if kind == 1 else
                 G.UnplacedSphere(5.0, 14.0) if kind == 2 else G.UnplacedTrd(6.0, 14.0, 20.0, 30.0, 25.0))
        lv = G.LogicalVolume("s%d" % k, solid)
        lv.SetMaterialPtr(1 + k % 2)
        lv.SetScored()
        angles = rng.uniform(0, 180, 3) if k % 2 else (0.0, 0.0, 0.0)
        world.PlaceDaughter("s%d" % k, lv, G.Transformation3D(x, y, z, *angles))
    gm = G.GeoManager()
    gm.SetWorld(world.Place())
    return gm.CloseGeometry()


class Tree:
    """point-in-solid by definition, for the checks"""

    def __init__(self, oracle, h):
        self.n, _ = oracle.csg_counts(h)
        self.nodes = [oracle.csg_node(h, i) for i in range(self.n)]

    def inside(self, geo, i, x):
        nd = self.nodes[i]
        R = np.array(nd["rotation"]).reshape(3, 3)
        q = R.T @ (x - np.array(nd["translation"]))
        s = geo.lv_solid[nd["lv"]]
        kind, (a, b, c) = geo.skind[s], geo.spar[s]
        if kind == 3:
            pl = geo.splanes[geo.splane_off[s]:geo.splane_off[s + 1]]
            n = pl[:, :3] / np.linalg.norm(pl[:, :3], axis=1, keepdims=True)
            return bool(np.all(n @ q < pl[:, 3] / np.linalg.norm(pl[:, :3], axis=1)))
        if kind == 0:
            return abs(q[0]) < a and abs(q[1]) < b and abs(q[2]) < c
        if kind == 1:
            r = math.hypot(q[0], q[1])
            if geo.splane_off[s + 1] > geo.splane_off[s]:  # a phi segment
                sphi, dphi = geo.splanes[geo.splane_off[s]][:2]
                if (math.atan2(q[1], q[0]) - sphi) % (2 * math.pi) >= dphi:
                    return False
            return a < r < b and abs(q[2]) < c if a > 0 else r < b and abs(q[2]) < c
        r = np.linalg.norm(q)
        return a < r < b if a > 0 else r < b

    def deepest(self, geo, x):
        if not self.inside(geo, 0, x):
            return -1
        v = 0
        while True:
            kids = [i for i in range(self.n) if self.nodes[i]["parent"] == v]
            nxt = [k for k in kids if self.inside(geo, k, x)]
            assert len(nxt) <= 1
            if not nxt:
                return v
            v = nxt[0]


def _rays(n, seed, targets, sigma=80.0):
    rng = np.random.default_rng(seed)
    # points near the solids (so that the rays meet them) and uniform directions
    centres = np.array(targets)
    p = centres[rng.integers(0, len(centres), n)] + rng.normal(0.0, sigma, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return p, d


def test_oracle_navigation_against_point_in_solid(oracle):
    geo = mixed_geometry()
    h = oracle.csg_build(geo)
    tree = Tree(oracle, h)
    assert tree.n == 1 + 1 + 1 + 2 * 4 + 2 + 2
    p, d = _rays(500, 11, [(100, -50, 20), (-250, 150, 0), (0, 350, -100), (-300, -300, 300), (250, 200, -200),
                           (200, -250, 250), (-100, -350, -300), (350, -50, 350)])
    vol, snext, nxt, saf = oracle.csg_probe(h, p, d)
    rng = np.random.default_rng(5)
    checked_hits = 0
    for i in range(len(p)):
        v = tree.deepest(geo, p[i])
        assert vol[i] == v, i
        if v < 0:
            continue
        s = snext[i]
        assert s > 0
        # the volume stays the same up to the boundary and changes after it
        for u in np.linspace(0.0, s - 1e-6, 64):
            assert tree.deepest(geo, p[i] + u * d[i]) == v, (i, u, s)
        assert tree.deepest(geo, p[i] + (s + 1e-6) * d[i]) == nxt[i], (i, s)
        checked_hits += nxt[i] != v
        # nothing but the current volume inside the safety sphere
        assert 0.0 <= saf[i] <= s + 1e-9
        if saf[i] > 1e-6:
            u = rng.normal(size=(32, 3))
            u /= np.linalg.norm(u, axis=1, keepdims=True)
            for x in p[i] + 0.999 * saf[i] * u:
                assert tree.deepest(geo, x) == v, i
    assert checked_hits > 150
    oracle.csg_free(h)


def test_oracle_limit_and_surface_direction(oracle):
    """children beyond the limit are not looked at; on a surface the
    direction decides the side"""
    from geantexascalepilot_b200 import geometry as G
    geo = G.calorimeter(axis=0)
    h = oracle.csg_build(geo)
    # on the Pb/LAr face of layer 0 (x = -197.7): moving +x is in LAr, -x in Pb
    face = -200.0 + 2.3
    vol, s, nxt, _ = oracle.csg_probe(h, [[face, 0, 0], [face, 0, 0]], [[1, 0, 0], [-1, 0, 0]])
    assert list(vol) == [3, 2] and np.allclose(s, [5.7, 2.3])
    assert list(nxt) == [5, -1]
    # a limit shorter than the distance: no crossing reported
    vol, s, nxt, _ = oracle.csg_probe(h, [[-199.0, 0, 0]], [[1, 0, 0]], limit=0.5)
    assert vol[0] == 2 and nxt[0] == 2 and s[0] >= 0.5
    oracle.csg_free(h)


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_oracle_tree_calorimeter_equals_layered(oracle, name):
    """The calorimeter built as a volume tree (layer volumes of two absorbers
    in a calorimeter volume, as the reference's detector construction) and
    the layered navigator: without a field the same tracks to rounding; in
    4 T the helix end points are relocated without the layered navigator's
    snap onto the plane, so a few tracks take other paths: statistics."""
    from geantexascalepilot_b200 import configs, geometry as G
    cfg, prims, nvol = configs.c2(16) if name == "c2" else configs.c3(8, 8)
    geo = G.calorimeter(axis=cfg.axis)
    h = oracle.csg_build(geo)
    a = oracle.transport(oracle_config(cfg), *prims[:4], nvol=nvol)
    oc = oracle_config(cfg)
    oc.geometry, oc.csg = 2, h
    b = oracle.transport(oc, *prims[:4], nvol=nvol)
    oracle.csg_free(h)
    assert b["errors"] == 0
    e0 = prims[1].sum()
    assert abs(b["edep"].sum() + b["escaped"] - e0) <= 1e-9 * e0
    if name == "c2":
        assert a["steps"] == b["steps"] and a["tracks"] == b["tracks"]
        assert np.array_equal(a["primary_steps"], b["primary_steps"])
        np.testing.assert_allclose(b["edep"], a["edep"], rtol=1e-9, atol=1e-12 * a["edep"].max())
    else:
        assert abs(a["steps"] - b["steps"]) <= 0.01 * a["steps"]
        la, lb = a["edep"].reshape(-1, 2).sum(1), b["edep"].reshape(-1, 2).sum(1)
        big = la > 0.002 * la.sum()
        assert np.all(np.abs(la - lb)[big] <= 5 * 0.2 / np.sqrt(16) * la[big] + 1e-3 * la.sum())


def test_library_builder_flattens_like_the_oracle(oracle):
    """gx_geom_* (host code of the library, no GPU needed) unrolls the tree
    into the same touchables, in the same order, with the same transforms"""
    geo = mixed_geometry()
    tl = geo.touchables()
    h = oracle.csg_build(geo)
    n, nscore = oracle.csg_counts(h)
    assert len(tl) == n and geo.ntouchables == n and geo.nscore == nscore
    for i, t in enumerate(tl):
        o = oracle.csg_node(h, i)
        assert (t["lv"], t["parent"], t["score"]) == (o["lv"], o["parent"], o["score"])
        assert t["translation"] == o["translation"] and t["rotation"] == o["rotation"]
    oracle.csg_free(h)
    from geantexascalepilot_b200 import geometry as G
    cal = G.calorimeter(axis=0, world_margin=10.0).touchables()
    scored = [t for t in cal if t["score"] >= 0]
    assert [t["score"] for t in scored] == list(range(100))
    assert [t["name"] for t in scored[:4]] == ["abs_0", "abs_1", "abs_0", "abs_1"]
    assert scored[2]["translation"][0] == pytest.approx(-200.0 + 8.0 + 1.15)


def test_library_builder_rejects_bad_trees():
    from geantexascalepilot_b200 import geometry as G
    from geantexascalepilot_b200._lib import GxError, lib
    h = C.c_void_p()
    assert lib.gx_geom_create(C.byref(h)) == 0
    s, lv, lv2 = C.c_int(), C.c_int(), C.c_int()
    assert lib.gx_geom_box(h, 1.0, 1.0, 0.0, C.byref(s)) != 0
    assert lib.gx_geom_tube(h, 2.0, 1.0, 1.0, C.byref(s)) != 0
    assert lib.gx_geom_box(h, 1.0, 1.0, 1.0, C.byref(s)) == 0
    assert lib.gx_geom_logical_volume(h, s.value, 7, 0, C.byref(lv)) != 0
    assert lib.gx_geom_logical_volume(h, s.value, 1, 0, C.byref(lv)) == 0
    assert lib.gx_geom_logical_volume(h, s.value, 1, 0, C.byref(lv2)) == 0
    t = (C.c_double * 3)(0, 0, 0)
    skew = (C.c_double * 9)(1, 0.1, 0, 0, 1, 0, 0, 0, 1)
    assert lib.gx_geom_place_daughter(h, lv.value, lv2.value, t, skew, None) != 0
    # a volume placed inside itself (through another) never closes
    assert lib.gx_geom_place_daughter(h, lv.value, lv2.value, t, None, None) == 0
    assert lib.gx_geom_place_daughter(h, lv2.value, lv.value, t, None, None) == 0
    nt, ns = C.c_int(), C.c_int()
    assert lib.gx_geom_close(h, lv.value, C.byref(nt), C.byref(ns)) != 0
    assert b"touchables" in lib.gx_last_error_string()
    lib.gx_geom_destroy(h)
    with pytest.raises(ValueError):
        G.UnplacedTube(0.0, 1.0, 1.0, 0.0, -1.0)
    h = C.c_void_p()
    assert lib.gx_geom_create(C.byref(h)) == 0
    assert lib.gx_geom_tube_segment(h, 0.0, 1.0, 1.0, 0.0, 0.0, C.byref(s)) != 0
    assert lib.gx_geom_tube_segment(h, 0.0, 1.0, 1.0, 0.5, 7.0, C.byref(s)) == 0  # 2 pi or more: the full tube
    lib.gx_geom_destroy(h)
    # polyhedra whose planes bound no finite volume: a slab open along z, a
    # pyramid without a base, contradictory planes
    open_prism = [[1, 0, 0, 1], [-1, 0, 0, 1], [0, 1, 0, 1], [0, -1, 0, 1]]
    pyramid = [[1, 0, 1, 0], [-1, 0, 1, 0], [0, 1, 1, 0], [0, -1, 1, 0]]
    empty = [[1, 0, 0, -1], [-1, 0, 0, -1], [0, 1, 0, 1], [0, -1, 0, 1], [0, 0, 1, 1], [0, 0, -1, 1]]
    for planes in (open_prism, pyramid, empty):
        h = C.c_void_p()
        assert lib.gx_geom_create(C.byref(h)) == 0
        arr = (C.c_double * (4 * len(planes)))(*[x for p in planes for x in p])
        assert lib.gx_geom_polyhedron(h, len(planes), arr, C.byref(s)) != 0
        assert b"finite volume" in lib.gx_last_error_string() or b"planes" in lib.gx_last_error_string()
        lib.gx_geom_destroy(h)
    with pytest.raises(GxError):
        G.CsgGeometry([0], [[1, 1, 1]], [0], [9], [0], [], [], [], [], 0).build()


def test_oracle_rejects_unbounded_polyhedra(oracle):
    from geantexascalepilot_b200 import geometry as G
    for planes in ([[1, 0, 0, 1], [-1, 0, 0, 1], [0, 1, 0, 1], [0, -1, 0, 1]],
                   [[1, 0, 1, 0], [-1, 0, 1, 0], [0, 1, 1, 0], [0, -1, 1, 0]]):
        world = G.LogicalVolume("w", G.UnplacedBox(10.0, 10.0, 10.0))
        world.PlaceDaughter("p", G.LogicalVolume("p", G.ConvexPolyhedron(planes)))
        gm = G.GeoManager()
        gm.SetWorld(world)
        assert not oracle.csg_build(gm.CloseGeometry())
