"""B200-native EM particle-transport step path (drop-in for the per-track
stepping of Geant-RnD/GeantExascalePilot).

The compute runs in hand-written sm_100a CUDA kernels in lib/libgxb200.so,
reached through the C ABI of include/gx_abi.h; this package is the host-side
mirror of the reference's interfaces over that ABI.
"""
from ._lib import DATA_DIR, EXPORTED, LIB_PATH, GxError  # noqa: F401
from .api import (ANNIHILATION, BETHE_HEITLER, BHABHA, ELECTRON, GAMMA, KLEIN_NISHINA, MODE_PHYSICS,  # noqa: F401
                  MODE_QUIRK, MOLLER, POSITRON, SAUTER_GAVRILA, SELTZER_BERGER, TABLES, ConstFieldHelixStepper,
                  MRG32k3a, ProxyAnnihilation, ProxyBetheHeitler, ProxyBhabhaScattering, ProxyBremsstrahlung,
                  ProxyCompton, ProxyConversion, ProxyDataManager, ProxyIonization, ProxyKleinNishina,
                  ProxyMollerScattering, ProxyPhotoElectric, ProxySauterGavrila, ProxySeltzerBerger, autotune,
                  cut_convert, default_config, egamma_gun, hepevt_load, hepevt_read, math_eval, pdg_to_type,
                  set_direction_xyz,
                  spot_gun, transport, transport_host, transport_noalloc, TrackSoA, gpil, propagate, along_step,
                  post_step, transport_tracks)
from . import configs, geometry, sharding  # noqa: F401
