"""The five benchmark workloads of the EM transport path, as transport
configurations plus seeded synthetic primaries (numpy arrays on the host).

C1  10 MeV photons into a 10 cm lead cube, no field, charged secondaries
    deposit locally (the reference's CPU-runnable case).
C2  1 GeV electrons into the 50-layer Pb/LAr calorimeter, no field.
C3  10 GeV electrons and 10 GeV photons along +x through the calorimeter
    (layers along x) in a 4 T field along z.
C4  2^16 primaries, one third each e-, e+, gamma, log-uniform 10 MeV..100 GeV,
    5 degree cone about +z from a 2 x 2 cm spot on the front face, 4 T.
C5  4096 events, Poisson(100) 10 GeV electrons each, 10 degree cone, 4 T,
    scored per event and layer.

Calorimeter: 50 layers of 2.3 mm Pb + 5.7 mm LAr, 400 x 400 mm transverse,
centred on the origin (the front face is at -200 mm on the layering axis).
C4's primaries and C5's directions come from the beam-spot gun
(gx_spot_gun_host: MRG32k3a stream 1 of the run seed, separate from the
transport substreams); C5's multiplicities are Poisson draws of numpy's
PCG64 seeded with 7.  C1-C3 are monoenergetic pencil beams.
"""
import numpy as np

from ._lib import TransportConfig, lib
import ctypes as C

GAMMA, ELECTRON, POSITRON = 0, 1, 2


def base_config(seed):
    cfg = TransportConfig()
    lib.gx_transport_config_default(C.byref(cfg))
    for k in range(6):
        cfg.seed[k] = float(seed)
    return cfg


def calorimeter(cfg, axis, Bz):
    cfg.geometry = 1
    cfg.axis = axis
    cfg.nlayers = 50
    cfg.t_abs = 2.3
    cfg.t_gap = 5.7
    cfg.half_trans = 200.0
    cfg.Bz = Bz
    return cfg


def c1(n=10000):
    cfg = base_config(12345)
    cfg.geometry = 0
    cfg.axis = 2
    cfg.box_half[:] = [50.0, 50.0, 50.0]
    cfg.box_centre[:] = [0.0, 0.0, 50.0]
    cfg.box_mat = 1
    cfg.charged_local = 1
    types = np.full(n, GAMMA, np.int32)
    E = np.full(n, 10.0)
    pos = np.zeros((n, 3))
    d = np.tile([0.0, 0.0, 1.0], (n, 1))
    return cfg, (types, E, pos, d, None), 1


def c2(n=10000):
    cfg = calorimeter(base_config(2024), 2, 0.0)
    pos = np.zeros((n, 3))
    pos[:, 2] = -200.0
    d = np.tile([0.0, 0.0, 1.0], (n, 1))
    return cfg, (np.full(n, ELECTRON, np.int32), np.full(n, 1000.0), pos, d, None), 100


def c3(n_e=10000, n_g=10000):
    cfg = calorimeter(base_config(2024), 0, 4.0)
    n = n_e + n_g
    types = np.concatenate([np.full(n_e, ELECTRON, np.int32), np.full(n_g, GAMMA, np.int32)])
    pos = np.zeros((n, 3))
    pos[:, 0] = -200.0
    d = np.tile([1.0, 0.0, 0.0], (n, 1))
    return cfg, (types, np.full(n, 10000.0), pos, d, None), 100


def c4(n=65536):
    from .api import spot_gun
    cfg = calorimeter(base_config(12345), 2, 4.0)
    types, E, pos, d = spot_gun(n, types=(ELECTRON, POSITRON, GAMMA), energy=(10.0, 1.0e5), cone_deg=5.0, axis=2,
                                centre=(0.0, 0.0, -200.0), half=(10.0, 10.0), seed=list(cfg.seed), stream=1,
                                device=False)
    return cfg, (types, E, pos, d, None), 100


def c5(nevents=4096, mean=100):
    from .api import spot_gun
    cfg = calorimeter(base_config(7), 2, 4.0)
    rng = np.random.default_rng(7)
    mult = rng.poisson(mean, nevents)
    n = int(mult.sum())
    events = np.repeat(np.arange(nevents, dtype=np.int32), mult)
    cfg.nevents = nevents
    types, E, pos, d = spot_gun(n, types=(ELECTRON,), energy=(1.0e4, 1.0e4), cone_deg=10.0, axis=2,
                                centre=(0.0, 0.0, -200.0), half=(0.0, 0.0), seed=list(cfg.seed), stream=1,
                                device=False)
    return cfg, (types, E, pos, d, events), 100


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}
