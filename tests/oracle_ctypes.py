"""ctypes front ends for the two CPU references of the tests (test infrastructure).

``Oracle`` wraps oracle/liboracle.so, the plain-C restatement of the
reference's transport path.  ``Reference`` wraps oracle/_ref/libgxref.so,
the reference's own code compiled in place (only present where a reference
checkout was available at build time; its table and Seltzer-Berger entry
points need the reference's data directory as working directory).
"""
import ctypes as C
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA_DIR = os.path.join(REPO, "geantexascalepilot_b200", "data")
ORACLE_SO = os.path.join(REPO, "oracle", "liboracle.so")
# the parity build: the same oracle with the elementary functions of the CUDA
# library's FP64 parity variant (gx_math.h), for track-by-track comparisons
ORACLE_GXM_SO = os.path.join(REPO, "oracle", "liboracle_gxm.so")
REF_SO = os.path.join(REPO, "oracle", "_ref", "libgxref.so")


def reference_root():
    """The reference checkout: $GX_REFERENCE_ROOT, else a directory named
    `reference` beside this repository."""
    return os.environ.get("GX_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference"))


REF_DATA_CWD = os.path.join(reference_root(), "source/Geant/proxy/test/BasicCpuTransport")

P = C.c_void_p
D = C.c_double
I = C.c_int
L = C.c_long


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def lp(a):
    return a.ctypes.data_as(C.POINTER(C.c_longlong))


class ModelParams(C.Structure):
    _fields_ = [("mode", I), ("Z", I), ("cut", D), ("density_factor", D), ("sb", P), ("data", P),
                ("charge", I)]


class Config(C.Structure):
    _fields_ = [("geometry", I), ("axis", I), ("nlayers", I), ("t_abs", D), ("t_gap", D),
                ("half_trans", D), ("box_half", D * 3), ("box_centre", D * 3), ("box_mat", I),
                ("Bz", D), ("charged_local", I), ("max_steps", I), ("seed", D * 6),
                ("first_substream", L), ("nthreads", I), ("score_events", I), ("msc", I),
                ("field_map", C.c_void_p), ("csg", C.c_void_p)]


MODEL_IDS = {"kn": 0, "sg": 1, "bh": 2, "sb": 3, "mb": 4, "bhabha": 5, "annih": 6}
# byte offsets of the SB tables inside gxo_data_t (computed from the struct layout)
_NTABLES, _NMAT = 20, 3
_PVEC_SIZE = 8 + 4 * 8 + 3 * 8  # n,type (2 ints) + 4 doubles + 3 pointers
_SB_SIZE = (32 + 57 + 57 * 32) * 8
_SB_OFF = _NTABLES * _NMAT * _PVEC_SIZE + (4 * _NMAT) * 8 * 2 + 12 * 8


class TracksStruct(C.Structure):
    _fields_ = [("n", I)] + [(f, P) for f in ("type", "status", "event", "primary", "volume", "pos", "dir", "ekin",
                                              "nil", "msc", "rng")]


class Tracks:
    """Tracks for the oracle in flat host arrays (pos, dir, nil n x 3; rng
    n x 6 MRG32k3a state doubles)."""

    def __init__(self, n):
        self.n = n
        for f in ("type", "status", "event", "primary", "volume"):
            setattr(self, f, np.zeros(n, np.int32))
        for f, shape in (("pos", (n, 3)), ("dir", (n, 3)), ("nil", (n, 3)), ("rng", (n, 6)), ("ekin", (n,)),
                         ("msc", (n,))):
            setattr(self, f, np.zeros(shape))

    @classmethod
    def from_soa(cls, d):
        """From TrackSoA.numpy() of the CUDA library's SoA."""
        n = len(d["type"])
        t = cls(n)
        for f in ("type", "status", "event", "primary", "volume"):
            getattr(t, f)[:] = d[f]
        t.pos[:] = np.stack([d["x"], d["y"], d["z"]], 1)
        t.dir[:] = np.stack([d["dx"], d["dy"], d["dz"]], 1)
        t.nil[:] = np.stack([d["nil0"], d["nil1"], d["nil2"]], 1)
        t.ekin[:] = d["ekin"]
        t.msc[:] = d["msc_range"]
        t.rng[:] = d["rng"].astype(np.float64)
        return t

    def struct(self):
        s = TracksStruct()
        s.n = self.n
        for f in ("type", "status", "event", "primary", "volume", "pos", "dir", "ekin", "nil", "msc", "rng"):
            setattr(s, f, getattr(self, f).ctypes.data)
        return s


class Oracle:
    def __init__(self, path=ORACLE_SO, datadir=DATA_DIR):
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: %s (run __graft_entry__.build())" % path)
        self.lib = lib = C.CDLL(path)
        lib.gxo_data_load.restype = P
        lib.gxo_data_load.argtypes = [C.c_char_p]
        lib.gxo_mrg_uniform_batch.argtypes = [I, I, C.POINTER(D), C.POINTER(D)]
        lib.gxo_mrg_substreams.argtypes = [C.POINTER(D), L, I, C.POINTER(D)]
        lib.gxo_mrg_advance_batch.argtypes = [I, C.POINTER(D), L, L]
        lib.gxo_mrg_init_stream_id.argtypes = [L, C.POINTER(D)]
        lib.gxo_mrg_next_stream.argtypes = [C.POINTER(D), C.POINTER(D)]
        lib.gxo_table_value_batch.argtypes = [P, I, I, I, C.POINTER(D), C.POINTER(D)]
        lib.gxo_table_invrange_batch.argtypes = [P, I, I, I, C.POINTER(D), C.POINTER(D)]
        lib.gxo_get_cut_value.restype = D
        lib.gxo_get_cut_value.argtypes = [P, I, I]
        lib.gxo_sb_value.restype = D
        lib.gxo_sb_value.argtypes = [P, D, D]
        lib.gxo_interact_batch.argtypes = [I, C.POINTER(ModelParams), I] + [C.POINTER(D)] * 6 + [
            C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(D), C.POINTER(D)]
        for f in ("gxo_kn_xs_per_atom", "gxo_mb_xs_per_atom"):
            getattr(lib, f).restype = D
            getattr(lib, f).argtypes = [D, D]
        lib.gxo_annih_xs_per_electron.restype = D
        lib.gxo_annih_xs_per_electron.argtypes = [D]
        lib.gxo_coulomb_factor.restype = D
        lib.gxo_coulomb_factor.argtypes = [D]
        lib.gxo_sg_photo_electron_energy.restype = D
        lib.gxo_sg_photo_electron_energy.argtypes = [P, I, D, I]
        lib.gxo_pe_xs_sandia.restype = D
        lib.gxo_pe_xs_sandia.argtypes = [P, I, D, D]
        lib.gxo_post_step_gpil.restype = D
        lib.gxo_post_step_gpil.argtypes = [C.POINTER(D), D, D, C.POINTER(D), C.POINTER(D)]
        lib.gxo_ioni_along_gpil.restype = D
        lib.gxo_ioni_along_gpil.argtypes = [P, I, I, I, D]
        lib.gxo_ioni_along_doit.argtypes = [P, I, I, I, D, C.POINTER(D), C.POINTER(D)]
        lib.gxo_helix_batch.argtypes = [C.POINTER(D), I] + [C.POINTER(D)] * 7
        lib.gxo_helix_dostep_mm.argtypes = [D] + [C.POINTER(D)] * 2 + [D, D, D] + [C.POINTER(D)] * 2
        lib.gxo_transport_flat.restype = I
        lib.gxo_transport_flat.argtypes = [P, C.POINTER(Config), I, C.POINTER(I), C.POINTER(D), C.POINTER(D),
                                           C.POINTER(D), C.POINTER(I), C.POINTER(D), I, C.POINTER(D),
                                           C.POINTER(C.c_longlong), C.POINTER(I)]
        lib.gxo_step_tracks.argtypes = [P, C.POINTER(Config), C.POINTER(TracksStruct), C.POINTER(TracksStruct),
                                        C.POINTER(D), I, C.POINTER(D), C.POINTER(C.c_longlong)]
        lib.gxo_transport_tracks.argtypes = [P, C.POINTER(Config), C.POINTER(TracksStruct), C.POINTER(D), I,
                                             C.POINTER(D), C.POINTER(C.c_longlong)]
        for f in ("gxo_gxm_eval", "gxo_libm_eval"):
            getattr(lib, f).argtypes = [I, I, C.POINTER(D), C.POINTER(D), C.POINTER(D)]
        self.data = lib.gxo_data_load(datadir.encode())
        if not self.data:
            raise RuntimeError("oracle could not load physics data from %s" % datadir)

    # --------------------------------------------- elementary functions
    MATH_FUNCS = {"log": 0, "exp": 1, "pow": 2, "sin": 3, "cos": 4, "expm1": 5, "log1p": 6}

    def math_eval(self, name, x, y=None, libm=False):
        """gx_math.h's function `name` (libm=False) or the C library's, at x
        (and y for pow)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, dtype=np.float64)
        out = np.zeros_like(x)
        f = self.lib.gxo_libm_eval if libm else self.lib.gxo_gxm_eval
        f(self.MATH_FUNCS[name], len(x), dp(x), dp(y), dp(out))
        return out

    # ------------------------------------------------------------ RNG
    def mrg_draws(self, states, k):
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6).copy()
        out = np.zeros((k, st.shape[0]))
        self.lib.gxo_mrg_uniform_batch(st.shape[0], k, dp(st), dp(out))
        return out, st

    def substreams(self, seed, first, n):
        s = np.ascontiguousarray(seed, dtype=np.float64)
        out = np.zeros((n, 6))
        self.lib.gxo_mrg_substreams(dp(s), first, n, dp(out))
        return out

    def advance(self, states, e, c):
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6).copy()
        self.lib.gxo_mrg_advance_batch(st.shape[0], dp(st), e, c)
        return st

    def stream_id_state(self, sid):
        s = np.zeros(6)
        self.lib.gxo_mrg_init_stream_id(sid, dp(s))
        return s

    # ----------------------------------------------------------- tables
    def table_value(self, table, mat, e):
        e = np.ascontiguousarray(e, dtype=np.float64)
        out = np.zeros_like(e)
        self.lib.gxo_table_value_batch(self.data, table, mat, e.size, dp(e), dp(out))
        return out

    def table_invrange(self, table, mat, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros_like(r)
        self.lib.gxo_table_invrange_batch(self.data, table, mat, r.size, dp(r), dp(out))
        return out

    def cut_value(self, index, ipart):
        return self.lib.gxo_get_cut_value(self.data, index, ipart)

    def sb_table_ptr(self, which):
        """which: 'slot10' (br11), 'ar' (br18), 'pb' (br82)"""
        k = {"slot10": 0, "ar": 1, "pb": 2}[which]
        return C.c_void_p(self.data + _SB_OFF + k * _SB_SIZE)

    def sb_value(self, which, x, y):
        return self.lib.gxo_sb_value(self.sb_table_ptr(which), x, y)

    # ----------------------------------------------------------- models
    def params(self, mode=0, Z=10, cut=0.0, density_factor=0.0, sb="slot10", charge=-1):
        return ModelParams(mode, Z, cut, density_factor, self.sb_table_ptr(sb), self.data, charge)

    def interact(self, model, states, E, dirs, params):
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6).copy()
        n = st.shape[0]
        E = np.ascontiguousarray(E, dtype=np.float64)
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(n, 3)
        out = dict(E=np.zeros(n), dir=np.zeros((n, 3)), edep=np.zeros(n), status=np.zeros(n, np.int32),
                   nsec=np.zeros(n, np.int32), sec_type=np.zeros((n, 2), np.int32), sec_E=np.zeros((n, 2)),
                   sec_dir=np.zeros((n, 2, 3)))
        self.lib.gxo_interact_batch(MODEL_IDS[model], C.byref(params), n, dp(st), dp(E), dp(dirs), dp(out["E"]),
                                    dp(out["dir"]), dp(out["edep"]), ip(out["status"]), ip(out["nsec"]),
                                    ip(out["sec_type"]), dp(out["sec_E"]), dp(out["sec_dir"]))
        out["states"] = st
        return out

    # ------------------------------------------------------- processes
    def post_step_gpil(self, state, lam, pstep_prev, nil, saved):
        st = np.ascontiguousarray(state, dtype=np.float64).copy()
        nil_c, saved_c = D(nil), D(saved)
        step = self.lib.gxo_post_step_gpil(dp(st), lam, pstep_prev, C.byref(nil_c), C.byref(saved_c))
        return step, nil_c.value, saved_c.value, st

    def ioni_along_gpil(self, mode, charge, mat, e):
        return self.lib.gxo_ioni_along_gpil(self.data, mode, charge, mat, e)

    def ioni_along_doit(self, mode, charge, mat, step, e):
        ec, ed = D(e), D(0.0)
        self.lib.gxo_ioni_along_doit(self.data, mode, charge, mat, step, C.byref(ec), C.byref(ed))
        return ec.value, ed.value

    def helix(self, B, pos, dirs, charge, mom, step):
        n = len(charge)
        B = np.ascontiguousarray(B, dtype=np.float64)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (pos, dirs, charge, mom, step)]
        npos, ndir = np.zeros((n, 3)), np.zeros((n, 3))
        self.lib.gxo_helix_batch(dp(B), n, *[dp(a) for a in args], dp(npos), dp(ndir))
        return npos, ndir

    # -------------------------------------------------------- transport
    def transport(self, cfg, types, E, pos, dirs, events=None, nvol=1, nevents=1):
        n = len(types)
        types = np.ascontiguousarray(types, dtype=np.int32)
        E = np.ascontiguousarray(E, dtype=np.float64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(n, 3)
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(n, 3)
        ev = np.ascontiguousarray(events if events is not None else np.zeros(n), dtype=np.int32)
        edep = np.zeros((nevents, nvol))
        esc = D(0.0)
        counters = np.zeros(9, dtype=np.int64)
        psteps = np.zeros(n, dtype=np.int32)
        rc = self.lib.gxo_transport_flat(self.data, C.byref(cfg), n, ip(types), dp(E), dp(pos), dp(dirs), ip(ev),
                                         dp(edep), nvol, C.byref(esc), lp(counters), ip(psteps))
        assert rc == 0
        names = ["steps", "substeps", "tracks", "sec_gamma", "sec_electron", "sec_positron", "n_pair", "n_annih",
                 "errors"]
        res = dict(zip(names, [int(c) for c in counters]))
        res.update(edep=edep, escaped=esc.value, primary_steps=psteps)
        return res

    def step_tracks(self, cfg, tracks, edep):
        """One OneStep of every alive track (in place); returns (secondaries
        Tracks at 2i, 2i+1, escaped energy, counters dict)."""
        sec = Tracks(2 * tracks.n)
        esc = D(0.0)
        counters = np.zeros(8, dtype=np.int64)
        ts, ss = tracks.struct(), sec.struct()
        self.lib.gxo_step_tracks(self.data, C.byref(cfg), C.byref(ts), C.byref(ss), dp(edep), edep.shape[-1],
                                 C.byref(esc), lp(counters))
        names = ["steps", "substeps", "sec_gamma", "sec_electron", "sec_positron", "n_pair", "n_annih", "errors"]
        return sec, esc.value, dict(zip(names, [int(c) for c in counters]))

    def transport_tracks(self, cfg, tracks, nvol, nevents=1):
        """The alive tracks of `tracks` to completion; returns a result dict
        like transport()'s."""
        edep = np.zeros((nevents, nvol))
        esc = D(0.0)
        counters = np.zeros(9, dtype=np.int64)
        ts = tracks.struct()
        assert self.lib.gxo_transport_tracks(self.data, C.byref(cfg), C.byref(ts), dp(edep), nvol, C.byref(esc),
                                             lp(counters)) == 0
        names = ["steps", "substeps", "tracks", "sec_gamma", "sec_electron", "sec_positron", "n_pair", "n_annih",
                 "errors"]
        res = dict(zip(names, [int(c) for c in counters]))
        res.update(edep=edep, escaped=esc.value)
        return res

    # ------------------------------------------------------------ field map
    def field_map_load(self, path):
        """load a map in the reference's CMS format; the handle goes into
        Config.field_map"""
        f = self.lib.gxo_field_map_load
        f.restype = C.c_void_p
        f.argtypes = [C.c_char_p]
        h = f(path.encode())
        assert h, path
        return h

    def field_map_value(self, handle, pos):
        f = self.lib.gxo_field_map_batch
        f.argtypes = [C.c_void_p, I, C.POINTER(D), C.POINTER(D)]
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        B = np.zeros_like(pos)
        f(handle, len(pos), dp(pos), dp(B))
        return B

    # --------------------------------------------------------- CSG geometry
    def csg_build(self, geo):
        """the oracle's flattened tree (gxo_csg_build) of a package
        CsgGeometry; the handle goes into Config.csg"""
        f = self.lib.gxo_csg_build
        f.restype = C.c_void_p
        f.argtypes = [I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, I, C.c_void_p, C.c_void_p, C.c_void_p, I,
                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, I]
        arrs = [np.ascontiguousarray(a) for a in (geo.skind, geo.spar, geo.splane_off, geo.splanes, geo.lv_solid,
                                                   geo.lv_mat, geo.lv_scored, geo.pv_mother, geo.pv_lv, geo.pv_t,
                                                   geo.pv_r)]
        self._keep = arrs
        v = [a.ctypes.data_as(C.c_void_p) for a in arrs]
        h = f(len(geo.skind), v[0], v[1], v[2], v[3], len(geo.lv_solid), v[4], v[5], v[6], len(geo.pv_mother), v[7],
              v[8], v[9], v[10], geo.world)
        return h

    def csg_free(self, h):
        self.lib.gxo_csg_free.argtypes = [C.c_void_p]
        self.lib.gxo_csg_free(h)

    def csg_counts(self, h):
        f = self.lib.gxo_csg_node_count
        f.argtypes = [C.c_void_p, C.POINTER(I)]
        ns = I()
        n = f(h, C.byref(ns))
        return n, ns.value

    def csg_node(self, h, i):
        f = self.lib.gxo_csg_node_info
        f.argtypes = [C.c_void_p, I, C.POINTER(I), C.POINTER(D)]
        info, tr = (I * 5)(), (D * 12)()
        f(h, i, info, tr)
        return dict(zip(("lv", "parent", "score", "mat", "nkid"), list(info)), translation=tuple(tr[:3]),
                    rotation=tuple(tr[3:]))

    def csg_probe(self, h, pos, dirs, limit=1e30):
        f = self.lib.gxo_csg_probe
        f.argtypes = [C.c_void_p, I] + [C.c_void_p] * 7
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        lim = np.ascontiguousarray(np.broadcast_to(np.asarray(limit, np.float64), (n,)))
        vol, nxt = np.zeros(n, np.int32), np.zeros(n, np.int32)
        snext, saf = np.zeros(n), np.zeros(n)
        f(h, n, *[a.ctypes.data_as(C.c_void_p) for a in (pos, dirs, lim, vol, snext, nxt, saf)])
        return vol, snext, nxt, saf

    def csg_contains(self, h, v, p, d, tol=1e-9):
        f = self.lib.gxo_csg_contains
        f.argtypes = [C.c_void_p, I, C.POINTER(D), C.POINTER(D), D]
        return bool(f(h, v, (D * 3)(*p), (D * 3)(*d), tol))

    # --------------------------------------------------- multiple scattering
    def material(self, Z, A, density):
        """gxo_material_t fields (Z, A, density, n_atoms, n_el, density_factor, radlen)"""
        buf = (D * 7)()
        self.lib.gxo_material_make.argtypes = [D, D, D, C.c_void_p]
        self.lib.gxo_material_make(Z, A, density, C.cast(buf, C.c_void_p))
        return dict(zip(("Z", "A", "density", "n_atoms", "n_el", "density_factor", "radlen"), list(buf)))

    def msc_cos(self, Z, X0, states, t, lam0, lam1, e0, e1):
        f = self.lib.gxo_msc_cos_batch
        f.argtypes = [D, D, I, C.POINTER(D)] + [D] * 5 + [C.POINTER(D)]
        st = np.ascontiguousarray(states, dtype=np.float64).copy()
        out = np.zeros(len(st))
        f(Z, X0, len(st), dp(st), t, lam0, lam1, e0, e1, dp(out))
        return out, st

    def msc_lambda1(self, type_, mat, e):
        f = self.lib.gxo_msc_lambda1
        f.restype = D
        f.argtypes = [P, I, I, D]
        return f(self.data, type_, mat, e)

    def msc_paths(self, t, lam):
        f, g = self.lib.gxo_msc_true_to_geom, self.lib.gxo_msc_geom_to_true
        f.restype = g.restype = D
        f.argtypes = [D, D]
        g.argtypes = [D, D, D]
        z = f(t, lam)
        return z, g(z, lam, t)

    # ------------------------------------------------------ event generators
    def egamma_gun(self, state, nevents, nparticles, gamma_fraction, minp, maxp, mineta, maxeta, minphi, maxphi):
        f = self.lib.gxo_egamma_gun
        f.restype = I
        f.argtypes = [C.POINTER(D), I, I] + [D] * 7 + [C.POINTER(I)] + [C.POINTER(D)] * 3
        st = np.ascontiguousarray(state, dtype=np.float64).copy()
        n = nevents * nparticles
        pdg = np.zeros(n, np.int32)
        p, ek, d = np.zeros(n), np.zeros(n), np.zeros((n, 3))
        k = f(dp(st), nevents, nparticles, gamma_fraction, minp, maxp, mineta, maxeta, minphi, maxphi, ip(pdg), dp(p),
              dp(ek), dp(d))
        assert k == n
        return pdg, p, ek, d, st

    def spot_gun(self, seed, stream, first, n, types, energy, cone_deg, axis, centre, half):
        f = self.lib.gxo_spot_gun
        f.argtypes = [C.POINTER(D), L, L, I, I, C.POINTER(I), D, D, D, I, C.POINTER(D), C.POINTER(D)] + \
            [C.c_void_p] * 4
        t, E = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1))
        pos, d = np.zeros((max(n, 1), 3)), np.zeros((max(n, 1), 3))
        f((D * 6)(*seed), stream, first, n, len(types), (I * 3)(*types), energy[0], energy[1], cone_deg, axis,
          (D * 3)(*centre), (D * 2)(*half), *[a.ctypes.data_as(C.c_void_p) for a in (t, E, pos, d)])
        return t[:n], E[:n], pos[:n], d[:n]

    def egamma_dir(self, physics, x, y, z):
        f = self.lib.gxo_egamma_dir
        f.argtypes = [I, D, D, D, C.POINTER(D), C.POINTER(D)]
        eta, phi = D(), D()
        f(physics, x, y, z, C.byref(eta), C.byref(phi))
        return eta.value, phi.value

    def hepevt(self, path, physics, max_events=1 << 30, cap=1 << 20):
        f = self.lib.gxo_hepevt_read
        f.restype = I
        f.argtypes = [C.c_char_p, I, I, I, C.POINTER(I), C.POINTER(I)] + [C.POINTER(D)] * 3 + [C.POINTER(I)] * 2
        ev, pdg = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        p, ek, d = np.zeros(cap), np.zeros(cap), np.zeros((cap, 3))
        nev, bad = C.c_int(), C.c_int()
        k = f(path.encode(), physics, max_events, cap, ip(ev), ip(pdg), dp(p), dp(ek), dp(d), C.byref(nev),
              C.byref(bad))
        assert k >= 0
        return dict(event=ev[:k], pdg=pdg[:k], p=p[:k], ekin=ek[:k], dir=d[:k], nevents=nev.value, bad=bad.value)


def oracle_config(cfg, nthreads=8):
    """The oracle's transport configuration for a package TransportConfig."""
    c = Config()
    for f in ("geometry", "axis", "nlayers", "t_abs", "t_gap", "half_trans", "box_mat", "Bz", "charged_local",
              "first_substream"):
        setattr(c, f, getattr(cfg, f))
    c.box_half[:] = list(cfg.box_half)
    c.box_centre[:] = list(cfg.box_centre)
    c.seed[:] = list(cfg.seed)
    c.max_steps = 10 ** 8
    c.nthreads = nthreads
    c.score_events = cfg.nevents
    c.msc = cfg.msc
    return c


class Reference:
    """The reference's own code (oracle/_ref/libgxref.so)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise RuntimeError("reference harness missing: %s" % path)
        self.lib = lib = C.CDLL(path)
        lib.gxref_mrg_draws.argtypes = [C.POINTER(D), I, C.POINTER(D), C.POINTER(D)]
        lib.gxref_mrg_stream_id.argtypes = [L, I, C.POINTER(D)]
        lib.gxref_mrg_advance.argtypes = [C.POINTER(D), L, L]
        lib.gxref_tables_init.restype = I
        for f in ("gxref_table_value", "gxref_table_invrange"):
            getattr(lib, f).restype = D
            getattr(lib, f).argtypes = [I, I, D]
        lib.gxref_cut_value.restype = D
        lib.gxref_cut_value.argtypes = [I, I]
        lib.gxref_sb2d_value.restype = D
        lib.gxref_sb2d_value.argtypes = [I, D, D]
        lib.gxref_interact.argtypes = [I, I] + [C.POINTER(D)] * 6 + [C.POINTER(I)] * 3 + [C.POINTER(D)] * 2
        for f in ("gxref_kn_xs", "gxref_mb_xs"):
            getattr(lib, f).restype = D
            getattr(lib, f).argtypes = [D, D]
        lib.gxref_sg_photo_energy.restype = D
        lib.gxref_sg_photo_energy.argtypes = [I, D]
        lib.gxref_coulomb.restype = D
        lib.gxref_coulomb.argtypes = [D]
        lib.gxref_post_step_gpil.restype = D
        lib.gxref_post_step_gpil.argtypes = [I, C.POINTER(D), D, D, C.POINTER(D), C.POINTER(D), I]
        lib.gxref_ioni_along_gpil.restype = D
        lib.gxref_ioni_along_gpil.argtypes = [I, D]
        lib.gxref_ioni_along_doit.argtypes = [I, D, C.POINTER(D), C.POINTER(D)]
        lib.gxref_helix.argtypes = [C.POINTER(D), I] + [C.POINTER(D)] * 7
        self._cwd_ready = False

    def _in_data_dir(self, fn, *a):
        old = os.getcwd()
        os.chdir(REF_DATA_CWD)
        try:
            return fn(*a)
        finally:
            os.chdir(old)

    def mrg_draws(self, seed, k):
        s = np.ascontiguousarray(seed, dtype=np.float64)
        out, st = np.zeros(k), np.zeros(6)
        self.lib.gxref_mrg_draws(dp(s), k, dp(out), dp(st))
        return out, st

    def stream_id_draws(self, sid, k):
        out = np.zeros(k)
        self.lib.gxref_mrg_stream_id(sid, k, dp(out))
        return out

    def advance(self, state, e, c):
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        self.lib.gxref_mrg_advance(dp(s), e, c)
        return s

    def init_tables(self):
        return self._in_data_dir(self.lib.gxref_tables_init)

    def table_value(self, table, mat, e):
        self.init_tables()
        return np.array([self.lib.gxref_table_value(table, mat, float(x)) for x in np.atleast_1d(e)])

    def table_invrange(self, table, mat, r):
        self.init_tables()
        return np.array([self.lib.gxref_table_invrange(table, mat, float(x)) for x in np.atleast_1d(r)])

    def cut_value(self, index, ipart):
        self.init_tables()
        return self.lib.gxref_cut_value(index, ipart)

    def sb2d_value(self, Z, x, y):
        return self._in_data_dir(self.lib.gxref_sb2d_value, Z, x, y)

    def interact(self, model, states, E, dirs):
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6).copy()
        n = st.shape[0]
        E = np.ascontiguousarray(E, dtype=np.float64)
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(n, 3)
        out = dict(E=np.zeros(n), dir=np.zeros((n, 3)), edep=np.zeros(n), status=np.zeros(n, np.int32),
                   nsec=np.zeros(n, np.int32), sec_type=np.zeros((n, 2), np.int32), sec_E=np.zeros((n, 2)),
                   sec_dir=np.zeros((n, 2, 3)))
        self._in_data_dir(self.lib.gxref_interact, MODEL_IDS[model], n, dp(st), dp(E), dp(dirs), dp(out["E"]),
                          dp(out["dir"]), dp(out["edep"]), ip(out["status"]), ip(out["nsec"]),
                          ip(out["sec_type"]), dp(out["sec_E"]), dp(out["sec_dir"]))
        out["states"] = st
        return out

    def post_step_gpil(self, process, state, e, pstep_prev, nil, saved, mat=2):
        self.init_tables()
        st = np.ascontiguousarray(state, dtype=np.float64).copy()
        nil_c, saved_c = D(nil), D(saved)
        step = self._in_data_dir(self.lib.gxref_post_step_gpil, process, dp(st), e, pstep_prev, C.byref(nil_c),
                                 C.byref(saved_c), mat)
        return step, nil_c.value, saved_c.value, st

    def ioni_along_gpil(self, mat, e):
        self.init_tables()
        return self._in_data_dir(self.lib.gxref_ioni_along_gpil, mat, e)

    def ioni_along_doit(self, mat, step, e):
        self.init_tables()
        ec, ed = D(e), D(0.0)
        self._in_data_dir(self.lib.gxref_ioni_along_doit, mat, step, C.byref(ec), C.byref(ed))
        return ec.value, ed.value

    def helix(self, B, pos, dirs, charge, mom, step):
        n = len(charge)
        B = np.ascontiguousarray(B, dtype=np.float64)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (pos, dirs, charge, mom, step)]
        npos, ndir = np.zeros((n, 3)), np.zeros((n, 3))
        self.lib.gxref_helix(dp(B), n, *[dp(a) for a in args], dp(npos), dp(ndir))
        return npos, ndir

    # ------------------------------------------------------ event generators
    def egamma_gun(self, state, nevents, nparticles, gamma_fraction, minp, maxp, mineta, maxeta, minphi, maxphi):
        f = self.lib.gxref_egamma_gun
        f.restype = I
        f.argtypes = [C.POINTER(D), I, I] + [D] * 7 + [C.POINTER(I)] + [C.POINTER(D)] * 3
        st = np.ascontiguousarray(state, dtype=np.float64).copy()
        n = nevents * nparticles
        pdg = np.zeros(n, np.int32)
        p, ek, d = np.zeros(n), np.zeros(n), np.zeros((n, 3))
        k = f(dp(st), nevents, nparticles, gamma_fraction, minp, maxp, mineta, maxeta, minphi, maxphi, ip(pdg), dp(p),
              dp(ek), dp(d))
        assert k == n
        return pdg, p, ek, d, st

    def egamma_direction(self, x, y, z):
        f = self.lib.gxref_egamma_direction
        f.argtypes = [D, D, D, C.POINTER(D)]
        d = np.zeros(3)
        f(x, y, z, dp(d))
        return d

    def hepevt(self, path, max_events, cap=1 << 16):
        f = self.lib.gxref_hepevt
        f.restype = I
        f.argtypes = [C.c_char_p, I, I, C.POINTER(I), C.POINTER(I)] + [C.POINTER(D)] * 3
        ev, pdg = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        p, ek, d = np.zeros(cap), np.zeros(cap), np.zeros((cap, 3))
        k = f(path.encode(), max_events, cap, ip(ev), ip(pdg), dp(p), dp(ek), dp(d))
        return dict(event=ev[:k], pdg=pdg[:k], p=p[:k], ekin=ek[:k], dir=d[:k])
