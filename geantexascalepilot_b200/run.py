"""Command-line transport of one benchmark workload on one GPU.

    python -m geantexascalepilot_b200.run c3 --electrons 2000 --photons 2000 --precision 1
    python -m geantexascalepilot_b200.run c5 --nevents 64 --mean 100 --profile
    python -m geantexascalepilot_b200.run c4 --n 4096 --autotune
    python -m geantexascalepilot_b200.run c3 --electrons 2000 --photons 2000 --profile --capacity 2097152
    python -m geantexascalepilot_b200.run c3 --geometry csg --msc 1 --field-map
    python -m geantexascalepilot_b200.run c3 --electrons 2000 --photons 2000 --iterations 30
    GX_LIB_PATH=geantexascalepilot_b200/lib/libgxb200_timeline.so \
        python -m geantexascalepilot_b200.run c3 --repeat 2 --timeline c3.npy

Prints one JSON line: the workload, the transport statistics (steps,
propagation sub-steps, tracks, secondaries, iterations, per-kernel device
times in profile mode) and the device time of the transport loop.  With
--iterations N the primaries go in as tracks (gx_transport_tracks) and the
engine stops after N iterations: the statistics are those of the first N
iterations, and the tracks still alive are handed back (their count is
printed); the difference of two such runs gives one iteration's work.
With --timeline FILE (the library's tracing build, see build.py) the last
repetition's per-iteration kernel timeline is saved to FILE (numpy) and
summarised in the JSON line.
"""
import argparse
import json
import sys


def main(argv=None):
    p = argparse.ArgumentParser(prog="python -m geantexascalepilot_b200.run")
    p.add_argument("workload", choices=["c1", "c2", "c3", "c4", "c5"])
    p.add_argument("--n", type=int, default=None, help="primaries (c1, c2, c4)")
    p.add_argument("--electrons", type=int, default=10000, help="c3")
    p.add_argument("--photons", type=int, default=10000, help="c3")
    p.add_argument("--nevents", type=int, default=4096, help="c5")
    p.add_argument("--mean", type=float, default=100.0, help="c5: mean primaries per event")
    p.add_argument("--precision", type=int, default=1, choices=[0, 1], help="0 FP64, 1 FP32-mixed")
    p.add_argument("--engine", type=int, default=1, choices=[0, 1], help="0 plain loop, 1 batched")
    p.add_argument("--profile", action="store_true", help="time each step kernel with CUDA events (no graph)")
    p.add_argument("--autotune", action="store_true", help="sweep the launch settings first")
    p.add_argument("--capacity", type=int, default=0,
                   help="track slots per particle type and store (0: the engine's default, 2^24)")
    p.add_argument("--repeat", type=int, default=1, help="transport the workload this many times")
    p.add_argument("--geometry", choices=["layers", "csg"], default="layers",
                   help="the analytic layered navigator, or the calorimeter as a CSG volume tree")
    p.add_argument("--msc", type=int, default=None, choices=[0, 1, 2],
                   help="multiple scattering: 0 off, 1 angular deflection, 2 with lateral displacement")
    p.add_argument("--field-map", action="store_true",
                   help="the shipped CMS field map (Runge-Kutta sub-steps) instead of the workload's uniform field")
    p.add_argument("--iterations", type=int, default=0,
                   help="stop after this many iterations and hand the live tracks back (0: run to completion)")
    p.add_argument("--timeline", default=None,
                   help="with the tracing build of the library: save the last repetition's kernel timeline here")
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)

    import torch

    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs

    torch.cuda.set_device(a.device)
    if a.workload == "c3":
        cfg, prims, nvol = configs.c3(a.electrons, a.photons)
    elif a.workload == "c5":
        cfg, prims, nvol = configs.c5(a.nevents, a.mean)
    else:
        fn = getattr(configs, a.workload)
        cfg, prims, nvol = fn(a.n) if a.n is not None else fn()
    cfg.precision, cfg.engine, cfg.profile = a.precision, a.engine, int(a.profile)
    cfg.capacity = a.capacity
    dm = gx.ProxyDataManager(device=a.device)
    out = {"workload": a.workload, "primaries": int(len(prims[0])), "precision": a.precision, "engine": a.engine}
    if a.geometry == "csg":
        from geantexascalepilot_b200 import geometry
        dm.load_geometry(geometry.calorimeter(axis=cfg.axis))
        cfg.geometry = 2
        out["geometry"] = "csg"
    if a.msc is not None:
        cfg.msc = a.msc
        out["msc"] = a.msc
    if a.field_map:
        dm.load_field_map()
        cfg.field_map = 1
        out["field_map"] = "cms"
    if a.autotune:
        cfg.profile = 0
        trials = gx.autotune(dm, cfg, *prims[:4], events=prims[4], nvol=nvol)
        out["autotune"] = trials[0]
        out["autotune_trials"] = trials
        cfg.profile = int(a.profile)
    for rep in range(a.repeat):
        if a.timeline and rep == a.repeat - 1:
            from geantexascalepilot_b200 import timeline
            torch.cuda.synchronize()
            timeline.reset(dm)
        if a.iterations > 0:
            tin = gx.TrackSoA.from_primaries(cfg, *prims[:4], events=prims[4])
            cap = min(4 * (a.capacity or (1 << 24)), 1 << 24)
            live, edep, st = gx.transport_tracks(dm, cfg, tin, max_iterations=a.iterations, out=gx.TrackSoA(cap),
                                                 nvol=nvol)
            out["iterations"] = a.iterations
            out["live_tracks"] = int(live.n)
        else:
            edep, st, _ = gx.transport(dm, cfg, *prims[:4], events=prims[4], nvol=nvol)
    torch.cuda.synchronize()
    if a.timeline:
        import numpy as np
        rec = timeline.read(dm)
        np.save(a.timeline, rec)
        out["timeline"] = timeline.summary(rec, st["iterations"])
    out["stats"] = st
    out["edep_total"] = float(edep.sum().item())
    out["track_steps_per_s"] = st["steps"] / (st["kernel_ms"] / 1e3) if st["kernel_ms"] > 0 else None
    print(json.dumps(out), flush=True)
    dm.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
