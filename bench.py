#!/usr/bin/env python3
"""Benchmark of the EM transport step path on B200.

One bench "step" is the complete transport of one batch of the headline
workload (C3: 10^4 electrons + 10^4 photons of 10 GeV through the 50-layer
Pb/LAr calorimeter in a 4 T field) with the FP32-mixed
batched engine.  `value` is track-steps/s over the timed steps with the
primaries already resident in HBM; `e2e` is the same metric through the
public host-buffer entry point (gx_transport_run_host), primaries copied in
and tallies copied out inside the timed region.  Beside it, the same batch on
the same MRG32k3a streams with the plain FP64 GPU loop and the batched FP64
engine, the per-layer energy-deposit difference FP32-mixed vs FP64, the
roofline of the dominant step kernel, and the CPU oracle timed on a bounded
sample on this machine's host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank transports its own batch (substreams offset by the
rank), so per-GPU work is fixed (weak scaling); the only collective is the
final sum of the per-layer tallies.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "track-steps/s on 1 B200: FP32-mixed vs FP64 GPU, ≤0.5% per-layer Edep diff"
UNIT = "track-steps/s"
LAUNCH_KEYS = ("block_size", "blocks_per_sm", "steps_per_launch", "graph_iters", "refill_below", "wave_energy")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="gx", choices=["gx", "reference"])
    p.add_argument("--electrons", type=int, default=10000)
    p.add_argument("--photons", type=int, default=10000)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison runs")
    p.add_argument("--autotune", action="store_true",
                   help="sweep the launch settings on the workload first (untimed) and time the winner")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- CPU side
def cpu_baseline(cfg_fn, seconds, nthreads):
    """Time the oracle's step loop on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from oracle_ctypes import Oracle
    from oracle_ctypes import oracle_config
    if not os.path.exists(os.path.join(REPO, "oracle", "liboracle.so")):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle")])
    orc = Oracle()
    n = 8
    while True:
        cfg, prims, nvol = cfg_fn(n)
        t0 = time.perf_counter()
        r = orc.transport(oracle_config(cfg, nthreads), *prims[:4], nvol=nvol)
        dt = time.perf_counter() - t0
        if dt >= seconds * 0.5 or n >= 20000:
            return r["steps"] / dt, n, dt
        n = int(min(20000, max(2 * n, n * seconds * 0.7 / max(dt, 1e-3))))


def c3_sample(ne, ng):
    from geantexascalepilot_b200 import configs
    return lambda n: configs.c3(n // 2 + n % 2, n // 2)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nth = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(c3_sample(args.electrons, args.photons), args.cpu_seconds / 4, nth)
    for _ in range(args.steps):
        v, n, dt = cpu_baseline(c3_sample(args.electrons, args.photons), args.cpu_seconds, nth)
        vals.append(v)
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "C3: 10 GeV e- + gamma, 50-layer Pb/LAr calorimeter, 4 T",
                                            "sample_primaries": n},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                             "sample": "%d C3 primaries (half e-, half gamma) per step, oracle step loop" % n},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU side
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs, geometry

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dm = gx.ProxyDataManager(device=local)
    cfg, prims, nvol = configs.c3(args.electrons, args.photons)
    nprim = len(prims[0])
    cfg.first_substream = rank * nprim
    types, E, pos, d, ev = prims
    dev = {"t": torch.as_tensor(types, device="cuda"), "E": torch.as_tensor(E, device="cuda"),
           "p": torch.as_tensor(pos, device="cuda"), "d": torch.as_tensor(d, device="cuda")}
    edep = torch.zeros((1, nvol), dtype=torch.float64, device="cuda")

    def one(precision, engine, profile=0, primary_steps=False):
        cfg.precision, cfg.engine, cfg.profile = precision, engine, profile
        edep.zero_()
        keep = [getattr(cfg, k) for k in LAUNCH_KEYS]
        if engine == 0:  # the plain loop runs with its own defaults
            for k in LAUNCH_KEYS:
                setattr(cfg, k, 0)
        try:
            _, st, ps = gx.transport(dm, cfg, dev["t"], dev["E"], dev["p"], dev["d"], nvol=nvol, edep=edep,
                                     primary_steps=primary_steps)
        finally:
            for k, v in zip(LAUNCH_KEYS, keep):
                setattr(cfg, k, v)
        return (st, ps.cpu().numpy()) if primary_steps else st

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def timed(precision, engine, steps, warmup):
        for _ in range(warmup):
            one(precision, engine)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_steps = 0
        launches = 0
        ev0.record()
        for _ in range(steps):
            st = one(precision, engine)
            n_steps += st["steps"]
            # per iteration: refill, refill_done, 3 transport, 8 interaction, finish; plain loop: 4
            launches += (14 if engine == 1 else 4) * (st["iterations"] + 1) + 3
        ev1.record()
        barrier()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = t.item()
            c = torch.tensor([n_steps], dtype=torch.float64, device="cuda")
            dist.all_reduce(c)
            n_steps = int(c.item())
        return ms, n_steps, launches, st

    tuned = None
    if args.autotune:
        cfg.precision, cfg.engine, cfg.profile = 1, 1, 0
        trials = gx.autotune(dm, cfg, dev["t"], dev["E"], dev["p"], dev["d"], nvol=nvol, repeats=2)
        tuned = {"best": trials[0], "trials": len(trials),
                 "default": next((t for t in trials if t["block_size"] == 128 and t["blocks_per_sm"] == 4
                                  and t["steps_per_launch"] == 16 and t["graph_iters"] == 16
                                  and t["wave_energy"] == 0), None)}

    # headline: FP32-mixed, batched engine, primaries resident in HBM
    with ClockSampler(local) as clk:
        ms, n_steps, launches, st32 = timed(1, 1, args.steps, args.warmup)
    e32 = edep.clone()
    value = n_steps / (ms / 1e3)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32-mixed (f64 rng/positions/boundaries/range-inversion)",
           "data": "synthetic",
           "config": {"workload": "C3: %d e- + %d gamma, 10 GeV, +x, 50 x (2.3 mm Pb + 5.7 mm LAr), 4 T along z"
                                  % (args.electrons, args.photons),
                      "engine": "batched (per-type queues, CUDA graph)", "parallelism": "replicas" if world > 1 else
                      "1 GPU", "l2": "track stores of several GB per step exceed L2 (no flush needed)"},
           "clocks": clk.summary(), "gpu_launches": launches,
           "track_steps_per_step": n_steps // max(1, args.steps), "primaries_per_s": world * nprim * args.steps / (ms / 1e3),
           "stats": {k: st32[k] for k in ("steps", "substeps", "tracks", "iterations", "peak_in_flight", "errors")},
           "launch": {"block": cfg.block_size or 128, "blocks_per_sm": cfg.blocks_per_sm or 4,
                      "steps_per_launch": cfg.steps_per_launch or 16,
                      "graph_iters": cfg.graph_iters or 16}}
    if tuned:
        out["autotune"] = tuned

    # FP64 comparisons on the same streams
    if not args.no_fp64:
        ms64p, s64p, _, _ = timed(0, 0, 1, 1)
        ms64b, s64b, _, _ = timed(0, 1, 1, 1)
        e64 = edep.clone()
        if world > 1:
            dist.all_reduce(e32)
            dist.all_reduce(e64)
        lay32 = e32.reshape(-1, 2).sum(1).cpu().numpy()
        lay64 = e64.reshape(-1, 2).sum(1).cpu().numpy()
        big = lay64 > 1e-3 * lay64.sum()
        rel = np.abs(lay32 - lay64)[big] / lay64[big]
        out["fp64_plain"] = {"value": s64p / (ms64p / 1e3), "unit": UNIT, "engine": "plain (one mixed queue, host loop)"}
        out["fp64_batched"] = {"value": s64b / (ms64b / 1e3), "unit": UNIT}
        out["speedup_vs_fp64_plain"] = value / out["fp64_plain"]["value"]
        out["layer_edep_rel_diff_fp32_vs_fp64"] = {"max": float(rel.max()), "mean": float(rel.mean()),
                                                   "total": float(abs(lay32.sum() - lay64.sum()) / lay64.sum()),
                                                   "layers_compared": int(big.sum())}
        # step-count distributions of the primaries, FP32-mixed vs FP64 (untimed runs)
        from scipy.stats import ks_2samp
        _, p32 = one(1, 1, primary_steps=True)
        _, p64 = one(0, 1, primary_steps=True)
        ks = ks_2samp(p32, p64)
        out["primary_step_count_ks_fp32_vs_fp64"] = {"statistic": float(ks.statistic), "pvalue": float(ks.pvalue),
                                                     "mean_fp32": float(p32.mean()), "mean_fp64": float(p64.mean())}

    # the same workload with multiple scattering of e-/e+ switched on
    # (Urban-type; the reference has none): FP32-mixed batched engine
    cfg.msc = 1
    msm, msteps, _, stm = timed(1, 1, 1, 1)
    cfg.msc = 0
    out["with_multiple_scattering"] = {"value": msteps / (msm / 1e3), "unit": UNIT, "steps": int(msteps),
                                       "substeps": int(stm["substeps"]), "ms": msm}

    # the other two throughput workloads on the same engine (FP32-mixed):
    # C4, 2^16 mixed e-/e+/gamma, log-uniform 10 MeV - 100 GeV, 4 T along z;
    # C5, 4096 events of Poisson(100) 10 GeV electrons scored per event
    # and C3 itself through the CSG volume tree (the calorimeter built from
    # placed boxes, as the reference's detector construction does)
    extra = {}
    for name, fn in (("c4", lambda: configs.c4(65536)), ("c5", lambda: configs.c5(4096, 100)),
                     ("c3_csg_tree", lambda: configs.c3())):
        c, pr, nv = fn()
        c.precision, c.engine, c.first_substream = 1, 1, rank * len(pr[0])
        if name == "c3_csg_tree":
            dm.load_geometry(geometry.calorimeter(axis=c.axis))
            c.geometry = 2
        tens = [torch.as_tensor(x, device="cuda") if x is not None else None for x in pr]
        gx.transport(dm, c, *tens[:4], events=tens[4], nvol=nv)  # warm-up
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, stx, _ = gx.transport(dm, c, *tens[:4], events=tens[4], nvol=nv)
        e1.record()
        barrier()
        msx = e0.elapsed_time(e1)
        extra[name] = {"track_steps_per_s": stx["steps"] / (msx / 1e3), "primaries_per_s": len(pr[0]) / (msx / 1e3),
                       "primaries": len(pr[0]), "steps": stx["steps"], "ms": msx}
        if name == "c5":
            extra[name]["events"] = int(c.nevents)
            extra[name]["events_per_s"] = c.nevents / (msx / 1e3)
    out["other_workloads"] = extra

    # e2e through the host-buffer entry point (warm-up calls first: the FP64
    # runs above released the FP32 engine's stores)
    # (inputs in page-locked host memory, as an application's staging buffers)
    cfg.precision, cfg.engine, cfg.profile = 1, 1, 0
    hp = [torch.as_tensor(np.ascontiguousarray(x)).pin_memory().numpy() for x in (types, E, pos, d)]
    for _ in range(args.warmup):
        gx.transport_host(dm, cfg, *hp, nvol=nvol)
    barrier()
    t0 = time.perf_counter()
    e2e_steps, calls = 0, []
    for _ in range(args.steps):
        tc = time.perf_counter()
        _, st = gx.transport_host(dm, cfg, *hp, nvol=nvol)
        calls.append({"ms": 1e3 * (time.perf_counter() - tc), "device_ms": st["kernel_ms"],
                      "iterations": st["iterations"]})
        e2e_steps += st["steps"]
    barrier()
    dt = time.perf_counter() - t0
    h2d = sum(x.nbytes for x in hp)
    out["e2e"] = {"value": world * e2e_steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                  "d2h_bytes_per_step": int(nvol * 8), "calls": calls}

    # roofline of the dominant kernel: the transport kernel of the particle type
    # that takes the most device time (profiling pass, CUDA events around each
    # launch on the launching stream)
    stp = one(1, 1, profile=1)
    k = int(np.argmax(stp["transport_ms"]))
    launches_k = max(1, stp["step_launches"][k])
    # algorithmic bytes: one read and one write of the track record per step
    # (a step reads and writes the state once); the kernel keeps a track in
    # registers across steps, so the records it actually moves are fewer
    nbytes = stp["transport_steps"][k] * 2 * stp["bytes_per_track"]
    moved = (stp["transport_read"][k] + stp["transport_written"][k]) * stp["bytes_per_track"]
    achieved = nbytes / (stp["transport_ms"][k] / 1e3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tr = os.path.join(REPO, "profiles", "transport_kernel_dram.txt")
    if os.path.exists(tr):
        # DRAM bytes per track record processed, from one ncu capture of this
        # kernel on a smaller case, scaled to this run's records per launch
        per = {}
        for line in open(tr):
            f = line.split()
            if len(f) == 2 and not line.startswith("#"):
                per[int(f[0])] = float(f[1])
        if k in per:
            traffic = per[k] * (stp["transport_read"][k] + stp["transport_written"][k]) / launches_k
    pipes = None
    pf = os.path.join(REPO, "profiles", "transport_kernel_pipes.txt")
    if os.path.exists(pf):
        # FP64 / FP32 / ALU pipe and issue utilisation (% of peak) of this
        # kernel from the same ncu capture: the kernel is latency-bound
        for line in open(pf):
            f = line.split()
            if len(f) == 6 and not line.startswith("#") and int(f[0]) == k:
                pipes = {"fp64_pct": float(f[1]), "fp32_fma_pct": float(f[2]), "alu_pct": float(f[3]),
                         "issue_pct": float(f[4]), "active_lanes_of_32": float(f[5]), "source": "ncu"}
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "traffic": traffic, "kernel": "k_transport<float,%d,0> (%s)" % (k, ["gamma", "e-", "e+"][k]),
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                       "algorithmic_bytes_per_launch": nbytes / launches_k,
                       "steps_per_launch": stp["transport_steps"][k] / launches_k,
                       "record_bytes_moved_per_launch": moved / launches_k,
                       "record_bytes_moved_gbs": moved / (stp["transport_ms"][k] / 1e3) / 1e9,
                       "avg_launch_ms": stp["transport_ms"][k] / launches_k,
                       "share_of_step_kernel_time": stp["transport_ms"][k] / max(1e-9, sum(stp["step_ms"])),
                       "records_per_launch": (stp["transport_read"][k] + stp["transport_written"][k]) / launches_k,
                       "pipes": pipes}

    if rank == 0:
        v, n, dtc = cpu_baseline(c3_sample(args.electrons, args.photons), args.cpu_seconds, os.cpu_count() or 1)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": "%d C3 primaries (half e-, half gamma), oracle step loop, %.1f s" % (n, dtc)}
        print(json.dumps(out), flush=True)
    dm.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
