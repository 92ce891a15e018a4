"""ctypes binding of libgxb200.so (the C ABI declared in include/gx_abi.h).

The library is the product: there is no fallback.  If it is missing the
import of the package raises, and every call checks the returned status and
raises ``GxError`` with the library's own message.
"""
import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GX_LIB_PATH") or os.path.join(PKG, "lib", "libgxb200.so")
DATA_DIR = os.path.join(PKG, "data")

GX_OK, GX_ERR_ARG, GX_ERR_CUDA, GX_ERR_DATA, GX_ERR_OVERFLOW, GX_ERR_ITERCAP, GX_ERR_NODEVICE = 0, -1, -2, -3, -4, -5, -6


class GxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("gx error %d: %s" % (code, msg))
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError("libgxb200.so is not built (%s); run __graft_entry__.build() or "
                      "python geantexascalepilot_b200/build.py" % LIB_PATH)

lib = C.CDLL(LIB_PATH)

P = C.c_void_p
I = C.c_int
D = C.c_double
LL = C.c_longlong
PD = C.POINTER(C.c_double)


class ModelParams(C.Structure):
    _fields_ = [("mode", I), ("Z", I), ("cut", D), ("density_factor", D), ("sb_table", I)]


class TransportConfig(C.Structure):
    _fields_ = [("geometry", I), ("axis", I), ("nlayers", I), ("t_abs", D), ("t_gap", D), ("half_trans", D),
                ("box_half", D * 3), ("box_centre", D * 3), ("box_mat", I), ("Bz", D), ("charged_local", I),
                ("max_steps", I), ("seed", D * 6), ("first_substream", LL), ("nevents", I), ("precision", I),
                ("engine", I), ("block_size", I), ("blocks_per_sm", I), ("capacity", LL), ("refill_below", LL),
                ("graph_iters", I), ("profile", I), ("wave_energy", D), ("steps_per_launch", I), ("msc", I),
                ("field_map", I), ("steps_per_launch_by_type", I * 3), ("interaction_interval", I),
                ("fp64_parity", I), ("fetch_min_by_type", I * 3)]


class TrackSoAStruct(C.Structure):
    """gx_track_soa (include/gx_abi.h): device pointers of the SoA fields."""
    _fields_ = ([("n", I), ("capacity", I)] +
                [(f, P) for f in ("type", "status", "event", "primary", "volume", "next_volume", "process",
                                  "boundary", "x", "y", "z", "dx", "dy", "dz", "ekin", "nil0", "nil1", "nil2",
                                  "lambda_inv0", "lambda_inv1", "lambda_inv2", "pstep", "step", "snext", "safety",
                                  "msc_range", "rng")])


class TransportStats(C.Structure):
    _fields_ = [("steps", LL), ("substeps", LL), ("tracks", LL), ("secondaries", LL * 3), ("n_pair", LL),
                ("n_annih", LL), ("errors", LL), ("escaped", D), ("iterations", LL), ("peak_in_flight", LL),
                ("kernel_ms", D), ("step_ms", D * 3), ("step_launches", LL * 3), ("tracks_read", LL * 3),
                ("tracks_written", LL * 3), ("bytes_per_track", LL), ("transport_ms", D * 3),
                ("transport_read", LL * 3), ("transport_written", LL * 3), ("transport_queued", LL * 3),
                ("transport_steps", LL * 3)]

    def as_dict(self):
        return {"steps": self.steps, "substeps": self.substeps, "tracks": self.tracks,
                "sec_gamma": self.secondaries[0], "sec_electron": self.secondaries[1],
                "sec_positron": self.secondaries[2], "n_pair": self.n_pair, "n_annih": self.n_annih,
                "errors": self.errors, "escaped": self.escaped, "iterations": self.iterations,
                "peak_in_flight": self.peak_in_flight, "kernel_ms": self.kernel_ms,
                "step_ms": list(self.step_ms), "step_launches": list(self.step_launches),
                "tracks_read": list(self.tracks_read), "tracks_written": list(self.tracks_written),
                "bytes_per_track": self.bytes_per_track, "transport_ms": list(self.transport_ms),
                "transport_read": list(self.transport_read), "transport_written": list(self.transport_written),
                "transport_queued": list(self.transport_queued), "transport_steps": list(self.transport_steps)}


class GunParams(C.Structure):
    _fields_ = [("nevents", I), ("nparticles", I), ("gamma_fraction", D), ("min_p", D), ("max_p", D),
                ("min_eta", D), ("max_eta", D), ("min_phi", D), ("max_phi", D), ("vertex", D * 3), ("seed", D * 6),
                ("first_draw", LL), ("first_event", I)]


class SpotGunParams(C.Structure):
    _fields_ = [("seed", D * 6), ("stream", LL), ("first", LL), ("ntypes", I), ("types", I * 3), ("emin", D),
                ("emax", D), ("cone_deg", D), ("axis", I), ("centre", D * 3), ("half", D * 2)]


AUTOTUNE_MAX_TRIALS = 64


class AutotuneReport(C.Structure):
    _fields_ = [("trials", I), ("best", I), ("block_size", I * AUTOTUNE_MAX_TRIALS),
                ("blocks_per_sm", I * AUTOTUNE_MAX_TRIALS), ("steps_per_launch", I * AUTOTUNE_MAX_TRIALS),
                ("graph_iters", I * AUTOTUNE_MAX_TRIALS),
                ("refill_below", LL * AUTOTUNE_MAX_TRIALS), ("wave_energy", D * AUTOTUNE_MAX_TRIALS),
                ("interaction_interval", I * AUTOTUNE_MAX_TRIALS),
                ("kernel_ms", D * AUTOTUNE_MAX_TRIALS), ("steps_per_ms", D * AUTOTUNE_MAX_TRIALS),
                ("fetch_min_gamma", I * AUTOTUNE_MAX_TRIALS)]

    def as_list(self):
        keys = ("block_size", "blocks_per_sm", "steps_per_launch", "graph_iters", "refill_below", "wave_energy",
                "interaction_interval", "fetch_min_gamma", "kernel_ms", "steps_per_ms")
        return [{k: getattr(self, k)[i] for k in keys} for i in range(self.trials)]


_SIGS = {
    "gx_last_error_string": (C.c_char_p, []),
    "gx_version": (I, []),
    "gx_ctx_create": (I, [C.c_char_p, I, C.POINTER(P)]),
    "gx_ctx_destroy": (I, [P]),
    "gx_rng_substreams": (I, [PD, LL, I, P, P]),
    "gx_rng_advance": (I, [P, I, LL, LL, P]),
    "gx_rng_uniform": (I, [P, I, I, P, P]),
    "gx_rng_stream_id": (I, [C.POINTER(LL), I, P, P]),
    "gx_table_value": (I, [P, I, I, P, P, I, P]),
    "gx_table_invrange": (I, [P, I, I, P, P, I, P]),
    "gx_sb_value": (I, [P, I, P, P, P, I, P]),
    "gx_cut_value": (I, [P, I, I, PD]),
    "gx_cut_convert": (I, [I, I, PD, PD, D, D, I, PD]),
    "gx_ctx_compute_cuts": (I, [P, D]),
    "gx_ctx_load_field_map": (I, [P, C.c_char_p]),
    "gx_field_value": (I, [P, I, P, P, P]),
    "gx_table_build": (I, [P, I, I, P, P, I, P]),
    "gx_ctx_rebuild_tables": (I, [P, PD]),
    "gx_interact": (I, [P, I, C.POINTER(ModelParams), I] + [P] * 11 + [P]),
    "gx_xs_per_atom": (I, [I, D, P, P, I, P]),
    "gx_post_step_gpil": (I, [P, I, I, I] + [P] * 6 + [P]),
    "gx_ioni_along_gpil": (I, [P, I, I, P, P, P, I, P]),
    "gx_ioni_along_doit": (I, [P, I, I, P, P, P, P, I, P]),
    "gx_helix_dostep": (I, [PD, D, I] + [P] * 15 + [P]),
    "gx_math_eval": (I, [I, I, I, P, P, P, P]),
    "gx_gpil": (I, [P, C.POINTER(TransportConfig), C.POINTER(TrackSoAStruct), P]),
    "gx_propagate": (I, [P, C.POINTER(TransportConfig), C.POINTER(TrackSoAStruct), P]),
    "gx_along_step": (I, [P, C.POINTER(TransportConfig), C.POINTER(TrackSoAStruct), P, I, P]),
    "gx_post_step": (I, [P, C.POINTER(TransportConfig), C.POINTER(TrackSoAStruct), C.POINTER(TrackSoAStruct), P, I,
                         P]),
    "gx_transport_tracks": (I, [P, C.POINTER(TransportConfig), C.POINTER(TrackSoAStruct), I,
                                C.POINTER(TrackSoAStruct), P, I, C.POINTER(TransportStats), P]),
    "gx_transport_config_default": (None, [C.POINTER(TransportConfig)]),
    "gx_transport_run": (I, [P, C.POINTER(TransportConfig), I, P, P, P, P, P, P, I, P, C.POINTER(TransportStats), P]),
    "gx_transport_run_host": (I, [P, C.POINTER(TransportConfig), I, P, P, P, P, P, P, I, P,
                                  C.POINTER(TransportStats)]),
    "gx_transport_autotune": (I, [P, C.POINTER(TransportConfig), I, P, P, P, P, P, I, I, C.POINTER(AutotuneReport),
                                  P]),
    "gx_timeline_reset": (I, [P]),
    "gx_timeline_read": (I, [P, P, LL]),
    "gx_egamma_gun": (I, [C.POINTER(GunParams), P, P, P, P, P, P, P]),
    "gx_pdg_to_type": (I, [I]),
    "gx_hepevt_read": (I, [C.c_char_p, I, I, I, P, P, P, P, C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
    "gx_hepevt_load": (I, [C.c_char_p, I, I, PD, I, P, P, P, P, P, C.POINTER(I), C.POINTER(I), C.POINTER(I), P]),
    "gx_transport_run_noalloc": (I, [P, C.POINTER(TransportConfig), I, P, P, P, P, P, P, I,
                                     C.POINTER(TransportStats), P]),
    "gx_spot_gun": (I, [C.POINTER(SpotGunParams), LL, P, P, P, P, P]),
    "gx_spot_gun_host": (I, [C.POINTER(SpotGunParams), LL, P, P, P, P]),
    "gx_geom_create": (I, [C.POINTER(P)]),
    "gx_geom_destroy": (None, [P]),
    "gx_geom_box": (I, [P, D, D, D, C.POINTER(I)]),
    "gx_geom_tube": (I, [P, D, D, D, C.POINTER(I)]),
    "gx_geom_tube_segment": (I, [P, D, D, D, D, D, C.POINTER(I)]),
    "gx_geom_sphere": (I, [P, D, D, C.POINTER(I)]),
    "gx_geom_polyhedron": (I, [P, I, PD, C.POINTER(I)]),
    "gx_geom_logical_volume": (I, [P, I, I, I, C.POINTER(I)]),
    "gx_geom_place_daughter": (I, [P, I, I, PD, PD, C.POINTER(I)]),
    "gx_geom_close": (I, [P, I, C.POINTER(I), C.POINTER(I)]),
    "gx_geom_touchable": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(I), PD, PD]),
    "gx_ctx_load_geometry": (I, [P, P]),
    "gx_geom_probe": (I, [P, I, P, P, P, P, P, P, P, P]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = sorted(_SIGS)


def check(rc):
    if rc != GX_OK:
        raise GxError(rc, lib.gx_last_error_string().decode(errors="replace"))
    return rc
