"""Host-side mirror of the reference's interfaces for the EM transport path.

Class and method names follow the reference (ProxyDataManager, MRG32k3a,
Proxy<Model>::SampleSecondaries, Proxy<Process>::PostStepGPIL,
ConstFieldHelixStepper::DoStepArr, ...) but every method works on a batch of
tracks held in torch CUDA tensors and calls the CUDA kernels through the C ABI
(include/gx_abi.h).  There is no CPU path: without a CUDA device the context
cannot be created and every call raises.
"""
import ctypes as C
import os

import numpy as np
import torch

from . import _lib
from ._lib import (AutotuneReport, GunParams, GxError, ModelParams, TrackSoAStruct, TransportConfig, TransportStats,
                   check, lib)

# physics-table ids (ProxyPhysicsTableIndex.hpp:23-45)
TABLES = ["DEDX.eBrem.e-", "DEDX.eBrem.e+", "DEDX.eIoni.e-", "DEDX.eIoni.e+", "InverseRange.eIoni.e-",
          "InverseRange.eIoni.e+", "Ionisation.eIoni.e-", "Ionisation.eIoni.e+", "Lambda.compt.gamma",
          "Lambda.conv.gamma", "Lambda.eBrem.e-", "Lambda.eBrem.e+", "Lambda.eIoni.e-", "Lambda.eIoni.e+",
          "LambdaMod1.msc.e-", "LambdaMod1.msc.e+", "LambdaPrim.compt.gamma", "LambdaPrim.phot.gamma",
          "Range.eIoni.e-", "Range.eIoni.e+"]
KLEIN_NISHINA, SAUTER_GAVRILA, BETHE_HEITLER, SELTZER_BERGER, MOLLER, BHABHA, ANNIHILATION = range(7)
MODE_QUIRK, MODE_PHYSICS = 0, 1
GAMMA, ELECTRON, POSITRON = 0, 1, 2


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(x, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(x, dtype=dtype, device="cuda").contiguous()


class ProxyDataManager:
    """Physics tables, cuts and Seltzer-Berger data on one device
    (ProxyDataManager, source/Geant/proxy/ProxyDataManager.cuh:27-83)."""

    def __init__(self, datadir=_lib.DATA_DIR, device=0):
        h = C.c_void_p()
        check(lib.gx_ctx_create(datadir.encode(), device, C.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib.gx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def table_build(self, table, mat, E):
        """A macroscopic cross-section table evaluated from the models
        (gx_table_build)."""
        E = _dev(E, torch.float64)
        out = torch.empty_like(E)
        check(lib.gx_table_build(self.handle, table, mat, _ptr(E), _ptr(out), E.numel(), _stream()))
        return out

    def rebuild_tables(self):
        """Replace the Compton, ionisation and e- brems tables by ones built
        from the models (gx_ctx_rebuild_tables); returns the largest relative
        change above 10 keV."""
        worst = C.c_double()
        check(lib.gx_ctx_rebuild_tables(self.handle, C.byref(worst)))
        return worst.value

    def load_field_map(self, path=None):
        """Load a field map in the reference's CMS format (gx_ctx_load_field_map);
        default: the CMS map shipped with the package."""
        import os
        path = path or os.path.join(_lib.DATA_DIR, "field", "cmsmagfield2015.txt")
        check(lib.gx_ctx_load_field_map(self.handle, path.encode()))

    def load_geometry(self, tree):
        """Upload a closed CSG volume tree (geometry.CsgGeometry, from
        GeoManager.CloseGeometry) for transport geometry 2
        (gx_ctx_load_geometry); returns its number of tally columns (nvol)."""
        return tree.load(self)

    def field_value(self, pos):
        """The loaded map's field (tesla) at positions (mm), shape (n, 3)."""
        p = _dev(pos, torch.float64).reshape(-1, 3).contiguous()
        B = torch.empty_like(p)
        check(lib.gx_field_value(self.handle, p.shape[0], _ptr(p), _ptr(B), _stream()))
        return B

    def compute_cuts(self, cut_mm=0.7):
        """Replace the cut table read from cut.dat by one converted from a
        range cut (gx_ctx_compute_cuts)."""
        check(lib.gx_ctx_compute_cuts(self.handle, cut_mm))

    # ProxyPhysicsTable::Value(index, E) of table `table`
    def table_value(self, table, mat, E):
        E = _dev(E, torch.float64)
        out = torch.empty_like(E)
        check(lib.gx_table_value(self.handle, table, mat, _ptr(E), _ptr(out), E.numel(), _stream()))
        return out

    # ProxyPhysicsVector::InvRangeValue
    def inv_range_value(self, table, mat, r):
        r = _dev(r, torch.float64)
        out = torch.empty_like(r)
        check(lib.gx_table_invrange(self.handle, table, mat, _ptr(r), _ptr(out), r.numel(), _stream()))
        return out

    # Proxy2DVector::Value on SB table 0 (br11), 1 (br18), 2 (br82)
    def sb_value(self, which, x, y):
        x = _dev(x, torch.float64)
        y = _dev(y, torch.float64)
        out = torch.empty_like(x)
        check(lib.gx_sb_value(self.handle, which, _ptr(x), _ptr(y), _ptr(out), x.numel(), _stream()))
        return out

    def GetCutValue(self, index, ipart):
        v = C.c_double()
        check(lib.gx_cut_value(self.handle, index, ipart, C.byref(v)))
        return v.value


class MRG32k3a:
    """Batches of MRG32k3a streams as (6, n) uint32 CUDA tensors
    (source/Geant/random/MRG32k3a.hpp)."""

    @staticmethod
    def substreams(seed, first, n):
        s = (C.c_double * 6)(*[float(v) for v in seed])
        out = torch.empty((6, n), dtype=torch.int32, device="cuda")
        check(lib.gx_rng_substreams(s, first, n, _ptr(out), _stream()))
        return out

    @staticmethod
    def from_states(states):
        """n x 6 array of the reference's FP64 words -> (6, n) device tensor"""
        t = torch.as_tensor(states, dtype=torch.float64).reshape(-1, 6).t().contiguous()
        return t.to(torch.int64).to(torch.int32).cuda()

    @staticmethod
    def to_states(t):
        """(6, n) device tensor -> n x 6 float64 CPU tensor of the six integers"""
        return (t.cpu().to(torch.int64) & 0xFFFFFFFF).to(torch.float64).t().contiguous()

    @staticmethod
    def uniform(states, k):
        n = states.shape[1]
        out = torch.empty((k, n), dtype=torch.float64, device="cuda")
        check(lib.gx_rng_uniform(_ptr(states), n, k, _ptr(out), _stream()))
        return out

    @staticmethod
    def advance(states, e, c):
        check(lib.gx_rng_advance(_ptr(states), states.shape[1], e, c, _stream()))
        return states

    @staticmethod
    def stream_id(ids):
        ids = list(ids)
        arr = (C.c_longlong * len(ids))(*ids)
        out = torch.empty((6, len(ids)), dtype=torch.int32, device="cuda")
        check(lib.gx_rng_stream_id(arr, len(ids), _ptr(out), _stream()))
        return out


class _Model:
    model_id = -1

    def __init__(self, dm, mode=MODE_QUIRK, Z=10, cut=0.0, density_factor=0.0, sb_table=0):
        self.dm = dm
        self.params = ModelParams(mode, Z, cut, density_factor, sb_table)

    def SampleSecondaries(self, E, direction, states):
        """ProxyEmModel<T>::SampleSecondaries for a batch; states are advanced."""
        E = _dev(E, torch.float64)
        d = _dev(direction, torch.float64).reshape(-1, 3)
        n = E.numel()
        o = {"E": torch.empty(n, dtype=torch.float64, device="cuda"),
             "dir": torch.empty((n, 3), dtype=torch.float64, device="cuda"),
             "edep": torch.empty(n, dtype=torch.float64, device="cuda"),
             "status": torch.empty(n, dtype=torch.int32, device="cuda"),
             "nsec": torch.empty(n, dtype=torch.int32, device="cuda"),
             "sec_type": torch.empty((n, 2), dtype=torch.int32, device="cuda"),
             "sec_E": torch.empty((n, 2), dtype=torch.float64, device="cuda"),
             "sec_dir": torch.empty((n, 2, 3), dtype=torch.float64, device="cuda")}
        check(lib.gx_interact(self.dm.handle, self.model_id, C.byref(self.params), n, _ptr(states), _ptr(E), _ptr(d),
                              _ptr(o["E"]), _ptr(o["dir"]), _ptr(o["edep"]), _ptr(o["status"]), _ptr(o["nsec"]),
                              _ptr(o["sec_type"]), _ptr(o["sec_E"]), _ptr(o["sec_dir"]), _stream()))
        return o

    def CrossSectionPerAtom(self, Z, E):
        E = _dev(E, torch.float64)
        out = torch.empty_like(E)
        check(lib.gx_xs_per_atom(self.model_id, float(Z), _ptr(E), _ptr(out), E.numel(), _stream()))
        return out


class ProxyKleinNishina(_Model):
    model_id = KLEIN_NISHINA


class ProxySauterGavrila(_Model):
    model_id = SAUTER_GAVRILA


class ProxyBetheHeitler(_Model):
    model_id = BETHE_HEITLER


class ProxySeltzerBerger(_Model):
    model_id = SELTZER_BERGER


class ProxyMollerScattering(_Model):
    model_id = MOLLER


class ProxyBhabhaScattering(_Model):
    model_id = BHABHA


class ProxyAnnihilation(_Model):
    model_id = ANNIHILATION


class _Process:
    process_id = -1

    def __init__(self, dm):
        self.dm = dm

    def PostStepGPIL(self, E, pstep_prev, nil, saved, states, mat=2):
        """ProxyEmProcess<T>::PostStepGPIL; nil and saved are updated in place."""
        E = _dev(E, torch.float64)
        ps = _dev(pstep_prev, torch.float64)
        step = torch.empty_like(E)
        check(lib.gx_post_step_gpil(self.dm.handle, self.process_id, mat, E.numel(), _ptr(states), _ptr(E), _ptr(ps),
                                    _ptr(nil), _ptr(saved), _ptr(step), _stream()))
        return step


class ProxyCompton(_Process):
    process_id = 0


class ProxyConversion(_Process):
    process_id = 1


class ProxyPhotoElectric(_Process):
    process_id = 2


class ProxyBremsstrahlung(_Process):
    process_id = 3


class ProxyIonization(_Process):
    process_id = 4

    def AlongStepGPIL(self, mat, E, mode=MODE_QUIRK, charge=-1):
        m = _dev(mat, torch.int32)
        E = _dev(E, torch.float64)
        out = torch.empty_like(E)
        check(lib.gx_ioni_along_gpil(self.dm.handle, mode, charge, _ptr(m), _ptr(E), _ptr(out), E.numel(), _stream()))
        return out

    def AlongStepDoIt(self, mat, step, E, mode=MODE_QUIRK, charge=-1):
        """returns (E after, energy deposited)"""
        m = _dev(mat, torch.int32)
        s = _dev(step, torch.float64)
        E = _dev(E, torch.float64).clone()
        edep = torch.zeros_like(E)
        check(lib.gx_ioni_along_doit(self.dm.handle, mode, charge, _ptr(m), _ptr(s), _ptr(E), _ptr(edep), E.numel(),
                                     _stream()))
        return E, edep


class ConstFieldHelixStepper:
    """ConstFieldHelixStepper (source/Geant/magneticfield/ConstFieldHelixStepper.hpp)."""

    def __init__(self, B, kB2C=-0.299792458e-3):
        self.B = (C.c_double * 3)(*[float(b) for b in B])
        self.kB2C = kB2C

    def DoStepArr(self, pos, direction, charge, momentum, step):
        pos = _dev(pos, torch.float64).reshape(-1, 3)
        d = _dev(direction, torch.float64).reshape(-1, 3)
        q = _dev(charge, torch.float64)
        p = _dev(momentum, torch.float64)
        s = _dev(step, torch.float64)
        n = q.numel()
        cols = [pos[:, k].contiguous() for k in range(3)] + [d[:, k].contiguous() for k in range(3)]
        outs = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(6)]
        check(lib.gx_helix_dostep(self.B, self.kB2C, n, *[_ptr(c) for c in cols], _ptr(q), _ptr(p), _ptr(s),
                                  *[_ptr(o) for o in outs], _stream()))
        return torch.stack(outs[:3], 1), torch.stack(outs[3:], 1)


# ------------------------------------------------------- tracks in SoA form
TRACK_ALIVE, TRACK_KILLED, TRACK_INTERACT, TRACK_EXITED = 0, 1, 2, 3


class TrackSoA:
    """A batch of tracks in SoA form (gx_track_soa): the hot fields of the
    reference's TrackState as the arrays of a TrackCollection
    (source/Geant/track/TrackState.hpp:30-232, TrackCollection.hpp:23-42),
    one CUDA tensor per field, `capacity` entries, the first `n` tracks.
    rng holds the MRG32k3a states as six planes of `capacity` uint32 words."""

    INT_FIELDS = ("type", "status", "event", "primary", "volume", "next_volume", "process", "boundary")
    DBL_FIELDS = ("x", "y", "z", "dx", "dy", "dz", "ekin", "nil0", "nil1", "nil2", "lambda_inv0", "lambda_inv1",
                  "lambda_inv2", "pstep", "step", "snext", "safety", "msc_range")

    def __init__(self, capacity, device="cuda"):
        self.capacity = int(capacity)
        self.n = 0
        for f in self.INT_FIELDS:
            setattr(self, f, torch.zeros(self.capacity, dtype=torch.int32, device=device))
        for f in self.DBL_FIELDS:
            setattr(self, f, torch.zeros(self.capacity, dtype=torch.float64, device=device))
        self.rng = torch.zeros(6 * self.capacity, dtype=torch.int32, device=device)

    @classmethod
    def from_primaries(cls, cfg, types, E, pos, direction, events=None, capacity=None, first_substream=None):
        """Primaries as tracks: stream = substream (first_substream + i) of
        cfg.seed (cfg.first_substream by default), NIL to be drawn, volume to
        be located -- the state gx_transport_run gives a primary."""
        n = len(types)
        t = cls(capacity or n)
        t.n = n
        t.type[:n] = torch.as_tensor(np.asarray(types), dtype=torch.int32)
        t.status[:n] = TRACK_ALIVE
        if events is not None:
            t.event[:n] = torch.as_tensor(np.asarray(events), dtype=torch.int32)
        t.primary[:n] = torch.arange(n, dtype=torch.int32)
        t.volume[:n] = -2
        p = np.asarray(pos, dtype=np.float64).reshape(n, 3)
        d = np.asarray(direction, dtype=np.float64).reshape(n, 3)
        for k, f in enumerate(("x", "y", "z")):
            getattr(t, f)[:n] = torch.as_tensor(p[:, k])
        for k, f in enumerate(("dx", "dy", "dz")):
            getattr(t, f)[:n] = torch.as_tensor(d[:, k])
        t.ekin[:n] = torch.as_tensor(np.asarray(E, dtype=np.float64))
        for f in ("nil0", "nil1", "nil2", "msc_range"):
            getattr(t, f)[:n] = -1.0
        first = cfg.first_substream if first_substream is None else first_substream
        st = torch.zeros(6 * n, dtype=torch.int32, device="cuda")
        check(lib.gx_rng_substreams((C.c_double * 6)(*cfg.seed), int(first), n, _ptr(st), _stream()))
        t.rng.view(6, t.capacity)[:, :n] = st.view(6, n)
        return t

    def struct(self):
        s = TrackSoAStruct()
        s.n, s.capacity = self.n, self.capacity
        for f in self.INT_FIELDS + self.DBL_FIELDS + ("rng",):
            setattr(s, f, getattr(self, f).data_ptr())
        return s

    def numpy(self):
        """The first n tracks as host arrays (rng as n x 6 uint32 words)."""
        n = self.n
        out = {f: getattr(self, f)[:n].cpu().numpy() for f in self.INT_FIELDS + self.DBL_FIELDS}
        out["rng"] = self.rng.view(6, self.capacity)[:, :n].cpu().numpy().view(np.uint32).T.copy()
        return out


def _stage(fn, dm, cfg, tracks, *extra):
    s = tracks.struct()
    check(fn(dm.handle, C.byref(cfg), C.byref(s), *extra))
    return s


def gpil(dm, cfg, tracks):
    """gx_gpil: PostStepGPIL of the discrete processes, range limit and
    FindNextBoundary for the ALIVE tracks (FP64; cfg.fp64_parity selects the
    parity variant)."""
    _stage(lib.gx_gpil, dm, cfg, tracks, _stream())


def propagate(dm, cfg, tracks):
    """gx_propagate: the move by the proposed step (straight or helix)."""
    _stage(lib.gx_propagate, dm, cfg, tracks, _stream())


def along_step(dm, cfg, tracks, edep):
    """gx_along_step: NIL update, continuous loss into edep [nevents, nvol],
    outcome of the step."""
    _stage(lib.gx_along_step, dm, cfg, tracks, _ptr(edep), edep.shape[1], _stream())


def post_step(dm, cfg, tracks, secondaries, edep):
    """gx_post_step: the interactions of the INTERACT tracks; secondaries of
    track i at entries 2i, 2i+1 of `secondaries` (capacity >= 2 n)."""
    t, sec = tracks.struct(), secondaries.struct()
    check(lib.gx_post_step(dm.handle, C.byref(cfg), C.byref(t), C.byref(sec), _ptr(edep), edep.shape[1],
                           _stream()))
    secondaries.n = sec.n


def transport_tracks(dm, cfg, tracks, max_iterations=0, out=None, edep=None, nvol=None):
    """gx_transport_tracks: the engine started from `tracks`, stopped after
    max_iterations iterations (0: to completion); returns (out TrackSoA with
    the tracks still alive, edep, stats)."""
    if nvol is None:
        nvol = 2 * cfg.nlayers if cfg.geometry == 1 else 1
    if edep is None:
        edep = torch.zeros((cfg.nevents, nvol), dtype=torch.float64, device="cuda")
    if out is None:
        out = TrackSoA(max(1024, 64 * max(1, tracks.n)))
    si, so = tracks.struct(), out.struct()
    st = TransportStats()
    check(lib.gx_transport_tracks(dm.handle, C.byref(cfg), C.byref(si), int(max_iterations), C.byref(so),
                                  _ptr(edep), nvol, C.byref(st), _stream()))
    out.n = so.n
    return out, edep, st.as_dict()


MATH_FUNCS = {"log": 0, "exp": 1, "pow": 2, "sin": 3, "cos": 4, "expm1": 5, "log1p": 6}


def math_eval(name, x, y=None, cuda_libm=False):
    """gx_math_eval: the FP64 parity variant's elementary function `name`
    (gx_math.h), or CUDA's own with cuda_libm, at the arguments x (and y for
    pow), on the device; returns a CUDA tensor."""
    xt = _dev(x, torch.float64)
    yt = _dev(y, torch.float64) if y is not None else None
    out = torch.empty_like(xt)
    check(lib.gx_math_eval(MATH_FUNCS[name], int(bool(cuda_libm)), xt.numel(), _ptr(xt), _ptr(yt), _ptr(out),
                           _stream()))
    return out


def default_config():
    cfg = TransportConfig()
    lib.gx_transport_config_default(C.byref(cfg))
    return cfg


def transport(dm, cfg, types, E, pos, direction, events=None, nvol=None, primary_steps=False, edep=None):
    """Transport primaries to completion (the reference's DoStep/OneStep loop).

    Inputs are CUDA tensors (or array-likes copied to the device).  Returns
    (edep [nevents, nvol] FP64 tensor, stats dict, per-primary step counts or None).
    """
    t = _dev(types, torch.int32)
    E = _dev(E, torch.float64)
    p = _dev(pos, torch.float64).reshape(-1, 3)
    d = _dev(direction, torch.float64).reshape(-1, 3)
    ev = _dev(events, torch.int32) if events is not None else None
    n = t.numel()
    if nvol is None:
        nvol = 2 * cfg.nlayers if cfg.geometry == 1 else 1
    if edep is None:
        edep = torch.zeros((cfg.nevents, nvol), dtype=torch.float64, device="cuda")
    ps = torch.zeros(n, dtype=torch.int32, device="cuda") if primary_steps else None
    st = TransportStats()
    check(lib.gx_transport_run(dm.handle, C.byref(cfg), n, _ptr(t), _ptr(E), _ptr(p), _ptr(d), _ptr(ev), _ptr(edep),
                               nvol, _ptr(ps), C.byref(st), _stream()))
    return edep, st.as_dict(), ps


def autotune(dm, cfg, types, E, pos, direction, events=None, nvol=None, repeats=2):
    """gx_transport_autotune: sweep the batched engine's launch settings on
    these primaries (the workload, or a representative subset), write the
    fastest into cfg and return the list of trials (best first)."""
    t = _dev(types, torch.int32)
    E = _dev(E, torch.float64)
    p = _dev(pos, torch.float64).reshape(-1, 3)
    d = _dev(direction, torch.float64).reshape(-1, 3)
    ev = _dev(events, torch.int32) if events is not None else None
    if nvol is None:
        nvol = 2 * cfg.nlayers if cfg.geometry == 1 else 1
    rep = AutotuneReport()
    check(lib.gx_transport_autotune(dm.handle, C.byref(cfg), t.numel(), _ptr(t), _ptr(E), _ptr(p), _ptr(d), _ptr(ev),
                                    nvol, repeats, C.byref(rep), _stream()))
    trials = rep.as_list()
    return [trials[rep.best]] + [x for i, x in enumerate(trials) if i != rep.best]


def transport_host(dm, cfg, types, E, pos, direction, events=None, nvol=None):
    """The same from host (numpy) buffers; copies happen inside the call."""
    import numpy as np
    t = np.ascontiguousarray(types, dtype=np.int32)
    E = np.ascontiguousarray(E, dtype=np.float64)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    d = np.ascontiguousarray(direction, dtype=np.float64)
    ev = np.ascontiguousarray(events, dtype=np.int32) if events is not None else None
    if nvol is None:
        nvol = 2 * cfg.nlayers if cfg.geometry == 1 else 1
    edep = np.zeros((cfg.nevents, nvol))
    st = TransportStats()
    vp = lambda a: C.c_void_p(a.ctypes.data) if a is not None else None  # noqa: E731
    check(lib.gx_transport_run_host(dm.handle, C.byref(cfg), t.size, vp(t), vp(E), vp(p), vp(d), vp(ev), vp(edep),
                                    nvol, None, C.byref(st)))
    return edep, st.as_dict()


def _abi_define(name):
    """An integer #define of include/gx_abi.h (the one place the limits live)."""
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "gx_abi.h")
    with open(hdr) as f:
        m = re.search(r"^#define\s+%s\s+(\d+)" % name, f.read(), re.M)
    if not m:
        raise RuntimeError("%s not defined in %s" % (name, hdr))
    return int(m.group(1))


NOALLOC_CAPACITY = _abi_define("GX_NOALLOC_CAPACITY")
NOALLOC_MAX_PRIMARIES = _abi_define("GX_NOALLOC_MAX_PRIMARIES")


def transport_noalloc(dm, cfg, types, E, pos, direction, events=None, nvol=None, edep=None):
    """gx_transport_run_noalloc: the plain FP64 loop on the library's static
    device array, for callers that cannot allocate device memory while they
    run (at most 4096 primaries, 16384 tracks in flight).  Inputs must already
    be CUDA tensors if the caller wants no allocation at all; array-likes are
    copied to the device here, by torch."""
    t = _dev(types, torch.int32)
    E = _dev(E, torch.float64)
    p = _dev(pos, torch.float64).reshape(-1, 3)
    d = _dev(direction, torch.float64).reshape(-1, 3)
    ev = _dev(events, torch.int32) if events is not None else None
    if nvol is None:
        nvol = 2 * cfg.nlayers if cfg.geometry == 1 else 1
    if edep is None:
        edep = torch.zeros((cfg.nevents, nvol), dtype=torch.float64, device="cuda")
    st = TransportStats()
    check(lib.gx_transport_run_noalloc(dm.handle, C.byref(cfg), t.numel(), _ptr(t), _ptr(E), _ptr(p), _ptr(d),
                                       _ptr(ev), _ptr(edep), nvol, C.byref(st), _stream()))
    return edep, st.as_dict()


# ------------------------------------------------------- primary generation
def egamma_gun(nevents, nparticles, gamma_fraction=0.5, momentum=(1.0e3, 1.0e6), eta=(-3.0, 3.0),
               phi=(0.0, 2.0 * 3.141592653589793), vertex=(0.0, 0.0, 0.0), seed=(12345.0,) * 6, first_draw=0,
               first_event=0):
    """ProxyEgammaGun (proxy/ProxyEgammaGun.hpp:35-82) on the device: returns
    CUDA tensors (types, E, pos, dir, events, pdg) ready for transport().
    Defaults are the reference's (1 GeV-1 TeV, |eta| < 3, full phi, seed
    12345 x 6, the stream a fresh ProxyRandom starts at)."""
    g = GunParams()
    g.nevents, g.nparticles, g.gamma_fraction = nevents, nparticles, gamma_fraction
    g.min_p, g.max_p = momentum
    g.min_eta, g.max_eta = eta
    g.min_phi, g.max_phi = phi
    g.vertex[:] = list(vertex)
    g.seed[:] = list(seed)
    g.first_draw, g.first_event = first_draw, first_event
    n = nevents * nparticles
    t = torch.empty(n, dtype=torch.int32, device="cuda")
    ev = torch.empty(n, dtype=torch.int32, device="cuda")
    pdg = torch.empty(n, dtype=torch.int32, device="cuda")
    E = torch.empty(n, dtype=torch.float64, device="cuda")
    pos = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    d = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    check(lib.gx_egamma_gun(C.byref(g), _ptr(t), _ptr(E), _ptr(pos), _ptr(d), _ptr(ev), _ptr(pdg), _stream()))
    return t, E, pos, d, ev, pdg


def _spot_params(n, types, energy, cone_deg, axis, centre, half, seed, stream, first):
    from ._lib import SpotGunParams
    g = SpotGunParams()
    g.seed[:] = [float(x) for x in seed]
    g.stream, g.first = stream, first
    g.ntypes = len(types)
    g.types[:len(types)] = list(types)
    g.emin, g.emax = energy
    g.cone_deg, g.axis = cone_deg, axis
    g.centre[:] = list(centre)
    g.half[:] = list(half)
    return g


def spot_gun(n, types=(ELECTRON, POSITRON, GAMMA), energy=(10.0, 1.0e5), cone_deg=5.0, axis=2,
             centre=(0.0, 0.0, -200.0), half=(10.0, 10.0), seed=(12345.0,) * 6, stream=1, first=0, device=True):
    """Beam-spot gun of the throughput workloads (gx_spot_gun): n primaries
    from MRG32k3a stream `stream` of the seed, five draws each (log-uniform
    kinetic energy in `energy`, direction in a cone about +axis, start on the
    spot centre +- half); types cycle through `types`.  Defaults: C4's.
    device=True returns CUDA tensors (types, E, pos, dir); device=False runs
    the host version (gx_spot_gun_host) into numpy arrays."""
    g = _spot_params(n, types, energy, cone_deg, axis, centre, half, seed, stream, first)
    if device:
        t = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        E = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
        pos = torch.empty((max(n, 1), 3), dtype=torch.float64, device="cuda")
        d = torch.empty((max(n, 1), 3), dtype=torch.float64, device="cuda")
        check(lib.gx_spot_gun(C.byref(g), n, _ptr(t), _ptr(E), _ptr(pos), _ptr(d), _stream()))
        return t[:n], E[:n], pos[:n], d[:n]
    t, E = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1))
    pos, d = np.zeros((max(n, 1), 3)), np.zeros((max(n, 1), 3))
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    check(lib.gx_spot_gun_host(C.byref(g), n, vp(t), vp(E), vp(pos), vp(d)))
    return t[:n], E[:n], pos[:n], d[:n]


def set_direction_xyz(x, y, z, mode=MODE_PHYSICS):
    """ProxyEgammaGun::SetDirectionXYZ (proxy/src/ProxyEgammaGun.cpp:35-41):
    the (eta, phi) both ranges collapse to.  MODE_QUIRK keeps the reference's
    theta = atan(rho / z) and phi = atan(y / z) (a beam along z gets an
    infinite eta, which the gun's range arithmetic turns into NaN, and z < 0
    a NaN eta);
    MODE_PHYSICS uses atan2 and keeps eta finite (|eta| <= 700: along the axis
    to within exp(-700))."""
    import math
    rho = math.sqrt(x * x + y * y)
    if mode == MODE_QUIRK:
        theta, ph = math.atan(rho / z), math.atan(y / z)
        t = math.tan(0.5 * theta)  # negative for z < 0: the reference's log gives NaN there
        return (-math.log(t) if t > 0 else (math.inf if t == 0 else math.nan)), ph
    theta, ph = math.atan2(rho, z), math.atan2(y, x)
    t = math.tan(0.5 * theta)
    eta = -math.log(t) if t > 0 else math.inf
    return max(-700.0, min(700.0, eta)), ph


def pdg_to_type(pdg):
    return lib.gx_pdg_to_type(int(pdg))


def hepevt_read(path, mode=MODE_PHYSICS, max_events=1 << 30):
    """ProxyHepEvtGenerator (proxy/src/ProxyHepEvtGenerator.cpp:48-132) on the
    host: dict of numpy arrays event, pdg, ekin (MeV in physics mode), dir,
    plus nevents and bad (daughter indices outside their event)."""
    import numpy as np
    n, nev, bad = C.c_int(), C.c_int(), C.c_int()
    rc = lib.gx_hepevt_read(path.encode(), mode, max_events, 0, None, None, None, None, C.byref(n), C.byref(nev),
                            C.byref(bad))
    if rc not in (_lib.GX_OK, _lib.GX_ERR_OVERFLOW):
        check(rc)
    cap = max(n.value, 1)
    ev, pdg = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    ek, d = np.zeros(cap), np.zeros((cap, 3))
    vp = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    check(lib.gx_hepevt_read(path.encode(), mode, max_events, cap, vp(ev), vp(pdg), vp(ek), vp(d), C.byref(n),
                             C.byref(nev), C.byref(bad)))
    k = n.value
    return {"event": ev[:k], "pdg": pdg[:k], "ekin": ek[:k], "dir": d[:k], "nevents": nev.value, "bad": bad.value}


def hepevt_load(path, mode=MODE_PHYSICS, max_events=1 << 30, vertex=(0.0, 0.0, 0.0), cap=None):
    """gx_hepevt_load: the gamma / e- / e+ primaries of a HEPEVT file in CUDA
    tensors (types, E, pos, dir, events), plus (nevents, nskipped)."""
    if cap is None:
        cap = len(hepevt_read(path, mode, max_events)["pdg"])
    t = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    ev = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    E = torch.empty(max(cap, 1), dtype=torch.float64, device="cuda")
    pos = torch.empty((max(cap, 1), 3), dtype=torch.float64, device="cuda")
    d = torch.empty((max(cap, 1), 3), dtype=torch.float64, device="cuda")
    vtx = (C.c_double * 3)(*vertex)
    n, nev, skip = C.c_int(), C.c_int(), C.c_int()
    check(lib.gx_hepevt_load(path.encode(), mode, max_events, vtx, cap, _ptr(t), _ptr(E), _ptr(pos), _ptr(d), _ptr(ev),
                             C.byref(n), C.byref(nev), C.byref(skip), _stream()))
    k = n.value
    return (t[:k], E[:k], pos[:k], d[:k], ev[:k]), (nev.value, skip.value)


def cut_convert(particle, Z, n_atoms, density, cut, from_length=True):
    """CutConverter::Convert (cuts/src/CutConverter.cpp:107-128) on the host:
    the energy (MeV) of a range cut (mm) for particle 0 gamma / 1 e- / 2 e+ in
    a material of elements Z with n_atoms per mm^3 and density g/cm^3, or the
    length of an energy cut when from_length is False."""
    Z = [float(z) for z in (Z if hasattr(Z, "__len__") else [Z])]
    n = [float(a) for a in (n_atoms if hasattr(n_atoms, "__len__") else [n_atoms])]
    out = C.c_double()
    check(lib.gx_cut_convert(particle, len(Z), (C.c_double * len(Z))(*Z), (C.c_double * len(n))(*n), density, cut,
                             1 if from_length else 0, C.byref(out)))
    return out.value

