"""CSG volume trees for transport geometry 2.

The classes take the calls a VecGeom detector construction makes, as the
reference's does (source/Geant/proxy/test/BasicCpuTransport/
ProxyDetectorConstruction.cpp:241-324): ``UnplacedBox`` / ``UnplacedTube`` /
``UnplacedSphere`` / ``UnplacedOrb`` / ``UnplacedTrd`` (and any convex
polyhedron given by its planes, ``ConvexPolyhedron``; tubes may be phi
segments), ``LogicalVolume`` with ``SetMaterialPtr`` and ``PlaceDaughter(name, lv, Transformation3D)``, and a
``GeoManager`` with ``SetWorld`` and ``CloseGeometry``.  Closing gives a
``CsgGeometry``: the tree as flat arrays, which ``load(dm)`` builds through the
C ABI (gx_geom_*) and uploads into a context.  Two additions: a material is an
index of the context's tables (0 G4_Galactic, 1 G4_Pb, 2 G4_lAr; the names are
accepted) and ``SetScored`` marks a logical volume whose placed instances get
tally columns, numbered depth-first from the world (the reference scores by
absorber logical volume and layer index instead).

Lengths are mm.  A placement puts a daughter point x at R x + t in its
mother; ``Transformation3D(tx, ty, tz, phi, theta, psi)`` takes the rotation
as Z-X-Z Euler angles in degrees, R = Rz(phi) Rx(theta) Rz(psi).
"""
import ctypes as C
import math

import numpy as np

from ._lib import check, lib

BOX, TUBE, SPHERE, POLY = 0, 1, 2, 3
MATERIALS = {"G4_Galactic": 0, "G4_Pb": 1, "G4_lAr": 2}


def _strip_name(args):
    return args[1:] if args and isinstance(args[0], str) else args


class UnplacedBox:
    kind = BOX

    def __init__(self, *args):
        """UnplacedBox([name,] hx, hy, hz): half lengths"""
        hx, hy, hz = _strip_name(args)
        self.par = (float(hx), float(hy), float(hz))


class UnplacedTube:
    kind = TUBE

    def __init__(self, *args):
        """UnplacedTube([name,] rmin, rmax, dz[, sphi, dphi]): phi in radians;
        dphi >= 2 pi (or no phi) is the full tube"""
        a = _strip_name(args)
        rmin, rmax, dz = a[:3]
        if len(a) not in (3, 5):
            raise ValueError("UnplacedTube: (rmin, rmax, dz) or (rmin, rmax, dz, sphi, dphi)")
        self.par = (float(rmin), float(rmax), float(dz))
        # the phi segment, None for the full tube
        self.phi = None if len(a) == 3 or a[4] >= 2 * math.pi else (float(a[3]), float(a[4]))
        if self.phi is not None and not self.phi[1] > 0.0:
            raise ValueError("UnplacedTube: dphi must be > 0")


class UnplacedSphere:
    kind = SPHERE

    def __init__(self, *args):
        """UnplacedSphere([name,] rmin, rmax[, sphi, dphi, stheta, dtheta]): full sphere only"""
        a = _strip_name(args)
        if len(a) > 2:
            full = len(a) == 6 and abs(a[3] - 2 * math.pi) < 1e-12 and a[4] == 0 and abs(a[5] - math.pi) < 1e-12
            if not full:
                raise ValueError("UnplacedSphere: only full spheres (shells) are supported")
        self.par = (float(a[0]), float(a[1]), 0.0)


class UnplacedOrb(UnplacedSphere):
    def __init__(self, *args):
        """UnplacedOrb([name,] r)"""
        (r,) = _strip_name(args)
        super().__init__(0.0, r)


class ConvexPolyhedron:
    """{x : n_k . x <= d_k}: planes as rows (nx, ny, nz, d), outward normals
    of any length (4 to 32 planes; they must bound a finite volume)"""
    kind = POLY

    def __init__(self, planes):
        self.planes = np.asarray(planes, np.float64).reshape(-1, 4)
        self.par = (0.0, 0.0, 0.0)


class UnplacedTrd(ConvexPolyhedron):
    def __init__(self, *args):
        """UnplacedTrd([name,] x1, x2, y1, y2, z): half lengths x1, y1 at -z and
        x2, y2 at +z, half length z along z"""
        a = _strip_name(args)
        if len(a) == 4:  # UnplacedTrd(x1, x2, y, z)
            a = (a[0], a[1], a[2], a[2], a[3])
        x1, x2, y1, y2, z = (float(v) for v in a)
        kx, ky = (x2 - x1) / (2.0 * z), (y2 - y1) / (2.0 * z)
        mx, my = 0.5 * (x1 + x2), 0.5 * (y1 + y2)
        # x <= mx + kx z, -x <= mx + kx z, and the same in y; |z| <= z
        super().__init__([[1.0, 0.0, -kx, mx], [-1.0, 0.0, -kx, mx], [0.0, 1.0, -ky, my], [0.0, -1.0, -ky, my],
                          [0.0, 0.0, 1.0, z], [0.0, 0.0, -1.0, z]])


def euler_zxz(phi, theta, psi):
    """R = Rz(phi) Rx(theta) Rz(psi), angles in degrees, row-major 9-tuple"""
    def rz(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])

    def rx(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])
    if phi == 0 and theta == 0 and psi == 0:
        return (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)
    R = rz(math.radians(phi)) @ rx(math.radians(theta)) @ rz(math.radians(psi))
    return tuple(float(x) for x in R.ravel())


class Transformation3D:
    def __init__(self, tx=0.0, ty=0.0, tz=0.0, phi=0.0, theta=0.0, psi=0.0):
        self.t = (float(tx), float(ty), float(tz))
        self.r = euler_zxz(phi, theta, psi)

    @classmethod
    def from_matrix(cls, translation, rotation):
        """a translation and a row-major (or 3 x 3) rotation matrix"""
        tr = cls(*translation)
        tr.r = tuple(float(x) for x in np.asarray(rotation, dtype=float).ravel())
        return tr


class PlacedVolume:
    def __init__(self, name, logical, transformation, mother):
        self.name, self.logical, self.transformation, self.mother = name, logical, transformation, mother

    def GetLogicalVolume(self):
        return self.logical


class LogicalVolume:
    def __init__(self, name, unplaced):
        self.name = name
        self.solid = unplaced
        self.material = 0
        self.scored = False
        self.daughters = []

    def SetMaterialPtr(self, material):
        self.material = MATERIALS[material] if isinstance(material, str) else int(material)

    def SetScored(self, scored=True):
        self.scored = bool(scored)

    def PlaceDaughter(self, name, logical, transformation=None):
        pv = PlacedVolume(name, logical, transformation or Transformation3D(), self)
        self.daughters.append(pv)
        return pv

    def Place(self, transformation=None):
        return PlacedVolume(self.name, self, transformation or Transformation3D(), None)


class GeoManager:
    def __init__(self):
        self.world = None

    def SetWorld(self, world):
        """the world's placed volume (LogicalVolume.Place()) or logical volume"""
        self.world = world.logical if isinstance(world, PlacedVolume) else world

    def GetWorld(self):
        return self.world

    def CloseGeometry(self):
        if self.world is None:
            raise ValueError("CloseGeometry: no world volume (SetWorld)")
        return CsgGeometry.from_tree(self.world)


class CsgGeometry:
    """A closed volume tree as flat arrays: solids (kind, 3 parameters),
    logical volumes (solid, material, scored), placements (mother and
    daughter logical volume, translation, rotation), the world's logical
    volume; the same arrays feed gx_geom_* and the oracle."""

    def __init__(self, skind, spar, lv_solid, lv_mat, lv_scored, pv_mother, pv_lv, pv_t, pv_r, world, names=None,
                 splane_off=None, splanes=None):
        self.skind = np.asarray(skind, np.int32)
        self.spar = np.asarray(spar, np.float64).reshape(-1, 3)
        # polyhedra: the planes of solid s are splanes[splane_off[s]:splane_off[s + 1]];
        # a tube with a phi segment has one row there, (sphi, dphi, 0, 0)
        self.splane_off = (np.zeros(len(self.skind) + 1, np.int32) if splane_off is None
                           else np.asarray(splane_off, np.int32))
        self.splanes = np.zeros((0, 4)) if splanes is None else np.asarray(splanes, np.float64).reshape(-1, 4)
        self.lv_solid = np.asarray(lv_solid, np.int32)
        self.lv_mat = np.asarray(lv_mat, np.int32)
        self.lv_scored = np.asarray(lv_scored, np.int32)
        self.pv_mother = np.asarray(pv_mother, np.int32)
        self.pv_lv = np.asarray(pv_lv, np.int32)
        self.pv_t = np.asarray(pv_t, np.float64).reshape(-1, 3)
        self.pv_r = np.asarray(pv_r, np.float64).reshape(-1, 9)
        self.world = int(world)
        self.names = names or ["lv%d" % i for i in range(len(self.lv_solid))]
        self.ntouchables = None
        self.nscore = None
        self._handle = None

    @classmethod
    def from_tree(cls, world):
        lvs, index = [], {}

        def visit(lv):
            if id(lv) in index:
                return
            index[id(lv)] = len(lvs)
            lvs.append(lv)
            for pv in lv.daughters:
                visit(pv.logical)
        visit(world)
        solids, sindex = [], {}
        for lv in lvs:
            if id(lv.solid) not in sindex:
                sindex[id(lv.solid)] = len(solids)
                solids.append(lv.solid)
        pv_mother, pv_lv, pv_t, pv_r = [], [], [], []
        for lv in lvs:
            for pv in lv.daughters:
                pv_mother.append(index[id(lv)])
                pv_lv.append(index[id(pv.logical)])
                pv_t.append(pv.transformation.t)
                pv_r.append(pv.transformation.r)
        off, planes = [0], []
        for s in solids:
            if s.kind == POLY:
                planes.extend(s.planes.tolist())
            elif s.kind == TUBE and getattr(s, "phi", None) is not None:
                planes.append([s.phi[0], s.phi[1], 0.0, 0.0])  # a tube's phi segment: (sphi, dphi)
            off.append(len(planes))
        return cls([s.kind for s in solids], [s.par for s in solids], [sindex[id(lv.solid)] for lv in lvs],
                   [lv.material for lv in lvs], [int(lv.scored) for lv in lvs], pv_mother, pv_lv,
                   np.array(pv_t).reshape(-1, 3), np.array(pv_r).reshape(-1, 9), 0, [lv.name for lv in lvs],
                   off, np.array(planes).reshape(-1, 4))

    # ------------------------------------------------------------ C ABI
    def build(self):
        """the tree through gx_geom_*; returns the builder handle (closed)"""
        h = C.c_void_p()
        check(lib.gx_geom_create(C.byref(h)))
        try:
            out = C.c_int()
            for s, (k, p) in enumerate(zip(self.skind, self.spar)):
                if k == POLY:
                    pl = np.ascontiguousarray(self.splanes[self.splane_off[s]:self.splane_off[s + 1]])
                    check(lib.gx_geom_polyhedron(h, len(pl), pl.ctypes.data_as(C.POINTER(C.c_double)),
                                                 C.byref(out)))
                elif k == BOX:
                    check(lib.gx_geom_box(h, p[0], p[1], p[2], C.byref(out)))
                elif k == TUBE and self.splane_off[s + 1] > self.splane_off[s]:
                    sphi, dphi = self.splanes[self.splane_off[s]][:2]
                    check(lib.gx_geom_tube_segment(h, p[0], p[1], p[2], sphi, dphi, C.byref(out)))
                elif k == TUBE:
                    check(lib.gx_geom_tube(h, p[0], p[1], p[2], C.byref(out)))
                else:
                    check(lib.gx_geom_sphere(h, p[0], p[1], C.byref(out)))
            for s, m, sc in zip(self.lv_solid, self.lv_mat, self.lv_scored):
                check(lib.gx_geom_logical_volume(h, int(s), int(m), int(sc), C.byref(out)))
            for mo, lv, t, r in zip(self.pv_mother, self.pv_lv, self.pv_t, self.pv_r):
                tt = (C.c_double * 3)(*t)
                rr = (C.c_double * 9)(*r)
                check(lib.gx_geom_place_daughter(h, int(mo), int(lv), tt, rr, C.byref(out)))
            nt, ns = C.c_int(), C.c_int()
            check(lib.gx_geom_close(h, self.world, C.byref(nt), C.byref(ns)))
        except Exception:
            lib.gx_geom_destroy(h)
            raise
        self.ntouchables, self.nscore = nt.value, ns.value
        return h

    def load(self, dm):
        """build and upload into the context of a ProxyDataManager; returns
        the number of tally columns (nvol for the transport)"""
        h = self.build()
        try:
            check(lib.gx_ctx_load_geometry(dm.handle, h))
        finally:
            lib.gx_geom_destroy(h)
        return self.nscore

    def touchables(self):
        """per touchable: logical volume, parent, tally column, translation, rotation"""
        h = self.build()
        try:
            out = []
            lv, par, sc = C.c_int(), C.c_int(), C.c_int()
            t, r = (C.c_double * 3)(), (C.c_double * 9)()
            for i in range(self.ntouchables):
                check(lib.gx_geom_touchable(h, i, C.byref(lv), C.byref(par), C.byref(sc), t, r))
                out.append({"lv": lv.value, "name": self.names[lv.value], "parent": par.value, "score": sc.value,
                            "translation": tuple(t), "rotation": tuple(r)})
            return out
        finally:
            lib.gx_geom_destroy(h)


def probe(dm, pos, direction, limit=1e30):
    """gx_geom_probe on the context's tree: (touchable, distance to the next
    boundary, touchable entered there, safety) per point, as CUDA tensors"""
    import torch
    from .api import _dev, _ptr, _stream
    p = _dev(pos, torch.float64).reshape(-1, 3)
    d = _dev(direction, torch.float64).reshape(-1, 3)
    n = p.shape[0]
    lim = _dev(np.broadcast_to(np.asarray(limit, np.float64), (n,)).copy() if not isinstance(limit, torch.Tensor)
               else limit, torch.float64)
    vol = torch.empty(n, dtype=torch.int32, device="cuda")
    nxt = torch.empty(n, dtype=torch.int32, device="cuda")
    snext = torch.empty(n, dtype=torch.float64, device="cuda")
    saf = torch.empty(n, dtype=torch.float64, device="cuda")
    check(lib.gx_geom_probe(dm.handle, n, _ptr(p), _ptr(d), _ptr(lim), _ptr(vol), _ptr(snext), _ptr(nxt), _ptr(saf),
                            _stream()))
    return vol, snext, nxt, saf


def calorimeter(axis=0, nlayers=50, t_abs=2.3, t_gap=5.7, half_trans=200.0, world_margin=0.0):
    """The Pb/LAr sampling calorimeter as a volume tree, built the way the
    reference's ProxyDetectorConstruction::CreateGeometry does (a layer volume
    holding the absorber and the gap, placed nlayers times in the calorimeter
    volume, placed in the world), layered along `axis`.  Absorber and gap are
    scored: tally column 2 layer + slab, as the layered navigator's.  With
    world_margin 0 the calorimeter is the world itself (a track leaving it
    escapes, as in the layered navigator)."""
    pitch = t_abs + t_gap

    def box(along, trans):
        h = [trans, trans, trans]
        h[axis] = along
        return UnplacedBox(*h)

    def at(x):
        t = [0.0, 0.0, 0.0]
        t[axis] = x
        return Transformation3D(*t)
    layer = LogicalVolume("layer", box(0.5 * pitch, half_trans))
    xstart = -0.5 * pitch
    for name, thick, mat in (("abs_0", t_abs, "G4_Pb"), ("abs_1", t_gap, "G4_lAr")):
        absor = LogicalVolume(name, box(0.5 * thick, half_trans))
        absor.SetMaterialPtr(mat)
        absor.SetScored()
        layer.PlaceDaughter(name, absor, at(xstart + 0.5 * thick))
        xstart += thick
    calo = LogicalVolume("calo", box(0.5 * nlayers * pitch, half_trans))
    xstart = -0.5 * nlayers * pitch
    for i in range(nlayers):
        calo.PlaceDaughter("layer_%d" % i, layer, at(xstart + 0.5 * pitch))
        xstart += pitch
    gm = GeoManager()
    if world_margin > 0.0:
        world = LogicalVolume("world", box(0.5 * nlayers * pitch + world_margin, half_trans + world_margin))
        world.PlaceDaughter("calorimeter", calo, Transformation3D())
        gm.SetWorld(world.Place())
    else:
        gm.SetWorld(calo.Place())
    return gm.CloseGeometry()
