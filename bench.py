#!/usr/bin/env python3
"""Benchmark of the EM transport step path on B200.

One bench "step" is the complete transport of one batch of the headline
workload (C3: 10^4 electrons + 10^4 photons of 10 GeV through the 50-layer
Pb/LAr calorimeter in a 4 T field) with the FP32-mixed batched engine.
`value` is track-steps/s over the timed steps with the primaries already
resident in HBM; `e2e` is the same metric through the public host-buffer entry
point (gx_transport_run_host), primaries copied in and tallies copied out
inside the timed region.  Beside it, on the same MRG32k3a streams:

  * the plain FP64 GPU loop and the batched FP64 engine (throughput);
  * the shower bar: per-layer energy deposit of FP32-mixed against the FP64
    GPU engine and against the CPU oracle (the reference's step loop restated
    and pinned to the reference's own code), each with its relative
    difference and its pull in standard deviations (sigma per layer from ten
    sub-batches of the batch, scored as ten events), and a KS test of the
    primaries' step counts;
  * the FP64 parity variant against the oracle's parity build on the whole
    batch: per-primary step counts and per-layer deposits;
  * C4 and C5 with the same arms (FP32-mixed, FP64 batched, FP64 plain loop
    -- C5 on a bounded sample of its events --, agreement, CPU sample), and
    C4 again at the setting gx_transport_autotune picks on a quarter of it;
  * the roofline of the dominant step kernel and the CPU oracle timed on the
    whole C3 batch on all host cores (the CPU baseline at equal statistics).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times the reference's CPU path (the oracle restatement,
built for this host) on the same C3 batch: the K timed steps are K slices of
the batch that together transport it once; it loads nothing of the CUDA
library.  Under torchrun each rank transports its own batch (substreams
offset by the rank), so per-GPU work is fixed (weak scaling); the only
collectives are the final sums of the tallies and the timing maximum.
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
LAUNCH_KEYS = ("block_size", "blocks_per_sm", "steps_per_launch", "graph_iters", "refill_below", "wave_energy",
               "interaction_interval")
NSUB = 10  # sub-batches of a batch for the per-layer standard deviations


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="gx", choices=["gx", "reference"])
    p.add_argument("--electrons", type=int, default=10000)
    p.add_argument("--photons", type=int, default=10000)
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU time of each bounded C4 / C5 oracle sample")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison runs")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle legs")
    p.add_argument("--no-tune-c4", action="store_true",
                   help="skip the launch-setting sweep on C4 (tuned on its first 16384 primaries)")
    p.add_argument("--autotune", action="store_true",
                   help="sweep the launch settings on the workload first (untimed) and time the winner")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def c3_config_dict(ne, ng):
    """The `config` of both arms' JSON lines (identical by construction)."""
    return {"workload": "C3: %d e- + %d gamma, 10 GeV, +x, 50 x (2.3 mm Pb + 5.7 mm LAr), 4 T along z" % (ne, ng),
            "primaries": ne + ng, "seed": "2024 x 6, substream = primary index",
            "l2": "track stores of several GB per step exceed L2 (no flush needed)"}


def c3_primaries(ne, ng):
    """C3's primaries (the same arrays as geantexascalepilot_b200.configs.c3,
    built here without the CUDA library)."""
    n = ne + ng
    types = np.concatenate([np.full(ne, 1, np.int32), np.full(ng, 0, np.int32)])
    pos = np.zeros((n, 3))
    pos[:, 0] = -200.0
    d = np.tile([1.0, 0.0, 0.0], (n, 1))
    return types, np.full(n, 1.0e4), pos, d


def c3_oracle_config(nthreads, nevents=1, first_substream=0):
    """The oracle's configuration of C3 (equal to oracle_config(configs.c3())),
    built without the CUDA library."""
    from oracle_ctypes import Config
    c = Config()
    c.geometry, c.axis, c.nlayers = 1, 0, 50
    c.t_abs, c.t_gap, c.half_trans, c.box_mat = 2.3, 5.7, 200.0, 1
    c.Bz, c.charged_local, c.first_substream = 4.0, 0, first_substream
    c.seed[:] = [2024.0] * 6
    c.max_steps = 10 ** 8
    c.nthreads = nthreads
    c.score_events = nevents
    c.msc = 0
    return c


def sub_batch_events(n, k=NSUB):
    """Primary i scores into event i % k: k sub-batches with the same mix of
    particle types."""
    return (np.arange(n) % k).astype(np.int32)


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
def load_oracle(parity=False):
    """The oracle built for this host (-O3 -march=native, `make native`), else
    the portable build; returns (Oracle, flags)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from oracle_ctypes import ORACLE_GXM_SO, ORACLE_SO, Oracle
    name = "liboracle_gxm.so" if parity else "liboracle.so"
    try:
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "native"], check=True, capture_output=True,
                       timeout=600)
        return Oracle(os.path.join(REPO, "oracle", "_native", name)), "gcc -O3 -march=native -ffp-contract=off"
    except (OSError, subprocess.SubprocessError):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle")])
        return Oracle(ORACLE_GXM_SO if parity else ORACLE_SO), "gcc -O3 -march=x86-64-v2 -ffp-contract=off"


def layer_sums(edep_events, nlayers=50):
    """[events, 2 nlayers] slab tally -> [events, nlayers] layer deposits."""
    e = np.asarray(edep_events)
    return e.reshape(e.shape[0], nlayers, 2).sum(2)


def total_and_sigma(per_sub):
    """Per-layer total over the sub-batches and its standard deviation
    (sqrt(k) times the spread of the k sub-batch values)."""
    k = per_sub.shape[0]
    return per_sub.sum(0), np.sqrt(k * per_sub.var(0, ddof=1))


def compare_layers(a, b, frac=0.002):
    """a, b: (total, sigma) per layer; layers holding > frac of b's deposit."""
    ta, sa = a
    tb, sb = b
    big = tb > frac * tb.sum()
    rel = np.abs(ta - tb)[big] / tb[big]
    pull = np.abs(ta - tb)[big] / np.sqrt(sa[big] ** 2 + sb[big] ** 2 + 1e-300)
    return {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "max_pull_sigma": float(pull.max()),
            "layers_compared": int(big.sum()), "total_rel": float(abs(ta.sum() - tb.sum()) / tb.sum()),
            "within_0.5pct_and_3sigma": bool(rel.max() <= 0.005 and pull.max() <= 3.0)}


def run_reference(args):
    """The reference arm: the oracle (the reference's CPU step loop restated,
    pinned to its own code) on all host cores, on the C3 batch the GPU arm
    transports; the K timed steps are K slices of it that together transport
    it once, the warm-up steps small slices of it."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nth = os.cpu_count() or 1
    orc, flags = load_oracle()
    types, E, pos, d = c3_primaries(args.electrons, args.photons)
    n = len(types)
    for w in range(args.warmup):
        sl = slice(w * 16, w * 16 + 16)
        orc.transport(c3_oracle_config(nth, first_substream=sl.start), types[sl], E[sl], pos[sl], d[sl], nvol=100)
    steps, t_total, edges = 0, 0.0, np.linspace(0, n, args.steps + 1).astype(int)
    per_step = []
    for k in range(args.steps):
        a, b = edges[k], edges[k + 1]
        t0 = time.perf_counter()
        r = orc.transport(c3_oracle_config(nth, first_substream=a), types[a:b], E[a:b], pos[a:b], d[a:b], nvol=100)
        dt = time.perf_counter() - t0
        steps += r["steps"]
        t_total += dt
        per_step.append(dt)
    v = steps / t_total
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": c3_config_dict(args.electrons, args.photons),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                             "sample": "the whole C3 batch (%d primaries, %d track-steps), transported once over the "
                                       "%d timed steps (consecutive slices of it); oracle step loop, %s, %d threads"
                                       % (n, steps, args.steps, flags, nth)},
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
    types, E, pos, d, _ = prims
    dev = {"t": torch.as_tensor(types, device="cuda"), "E": torch.as_tensor(E, device="cuda"),
           "p": torch.as_tensor(pos, device="cuda"), "d": torch.as_tensor(d, device="cuda")}
    edep = torch.zeros((1, nvol), dtype=torch.float64, device="cuda")

    def one(precision, engine, profile=0, primary_steps=False, parity=0, c=None, tens=None, events=None,
            out=None):
        c = cfg if c is None else c
        tens = dev if tens is None else tens
        out = edep if out is None else out
        c.precision, c.engine, c.profile, c.fp64_parity = precision, engine, profile, parity
        out.zero_()
        keep = [getattr(c, k) for k in LAUNCH_KEYS]
        if engine == 0:  # the plain loop runs with its own defaults
            for k in LAUNCH_KEYS:
                setattr(c, k, 0)
        try:
            _, st, ps = gx.transport(dm, c, tens["t"], tens["E"], tens["p"], tens["d"], events=events,
                                     nvol=out.shape[1], edep=out, primary_steps=primary_steps)
        finally:
            for k, v in zip(LAUNCH_KEYS, keep):
                setattr(c, k, v)
            c.fp64_parity = 0
        return (st, ps.cpu().numpy()) if primary_steps else st

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def timed(precision, engine, steps, warmup, parity=0, c=None, tens=None, events=None, out=None):
        for _ in range(warmup):
            one(precision, engine, parity=parity, c=c, tens=tens, events=events, out=out)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_steps = 0
        launches = 0
        ev0.record()
        for _ in range(steps):
            st = one(precision, engine, parity=parity, c=c, tens=tens, events=events, out=out)
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
            c_ = torch.tensor([n_steps], dtype=torch.float64, device="cuda")
            dist.all_reduce(c_)
            n_steps = int(c_.item())
        return ms, n_steps, launches, st

    tuned = None
    if args.autotune:
        cfg.precision, cfg.engine, cfg.profile = 1, 1, 0
        trials = gx.autotune(dm, cfg, dev["t"], dev["E"], dev["p"], dev["d"], nvol=nvol, repeats=2)
        tuned = {"best": trials[0], "trials": len(trials),
                 "default": next((t for t in trials if t["block_size"] == 128 and t["blocks_per_sm"] == 5
                                  and t["steps_per_launch"] == 16 and t["graph_iters"] == 16
                                  and t["wave_energy"] == 0), None)}

    # headline: FP32-mixed, batched engine, primaries resident in HBM
    with ClockSampler(local) as clk:
        ms, n_steps, launches, st32 = timed(1, 1, args.steps, args.warmup)
    value = n_steps / (ms / 1e3)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32-mixed (f64 rng/positions/boundaries/range-inversion)",
           "data": "synthetic", "config": c3_config_dict(args.electrons, args.photons),
           "engine": "batched (per-type queues, CUDA graph), " + ("replicas" if world > 1 else "1 GPU"),
           "clocks": clk.summary(), "gpu_launches": launches,
           "track_steps_per_step": n_steps // max(1, args.steps),
           "primaries_per_s": world * nprim * args.steps / (ms / 1e3),
           "stats": {k: st32[k] for k in ("steps", "substeps", "tracks", "iterations", "peak_in_flight", "errors")},
           "launch": {"block": cfg.block_size or 128, "blocks_per_sm": cfg.blocks_per_sm or 5,
                      "steps_per_launch": cfg.steps_per_launch or 16,
                      "graph_iters": cfg.graph_iters or 16}}
    if tuned:
        out["autotune"] = tuned

    # C3 in ten sub-batches (primary i scores into event i % 10) for the
    # per-layer standard deviations; untimed, the same streams as above
    ev_np = sub_batch_events(nprim)
    ev_t = torch.as_tensor(ev_np, device="cuda")
    cfg.nevents = NSUB
    sub_edep = torch.zeros((NSUB, nvol), dtype=torch.float64, device="cuda")
    layers = {}
    _, p32 = one(1, 1, primary_steps=True, events=ev_t, out=sub_edep)
    layers["fp32"] = layer_sums(sub_edep.cpu().numpy())
    if not args.no_fp64:
        _, p64 = one(0, 1, primary_steps=True, events=ev_t, out=sub_edep)
        layers["fp64"] = layer_sums(sub_edep.cpu().numpy())
        _, ppar = one(0, 1, primary_steps=True, parity=1, events=ev_t, out=sub_edep)
        layers["fp64_parity"] = layer_sums(sub_edep.cpu().numpy())
    cfg.nevents = 1

    # FP64 comparisons on the same streams (throughput)
    if not args.no_fp64:
        ms64p, s64p, _, _ = timed(0, 0, 1, 1)
        ms64b, s64b, _, _ = timed(0, 1, 1, 1)
        msx, sx, _, _ = timed(0, 1, 1, 1, parity=1)
        out["fp64_plain"] = {"value": s64p / (ms64p / 1e3), "unit": UNIT, "engine": "plain (one mixed queue, host loop)"}
        out["fp64_batched"] = {"value": s64b / (ms64b / 1e3), "unit": UNIT}
        out["fp64_parity_batched"] = {"value": sx / (msx / 1e3), "unit": UNIT,
                                      "note": "the FP64 parity variant: no FMA contraction, gx_math.h functions"}
        out["speedup_vs_fp64_plain"] = value / out["fp64_plain"]["value"]
        out["speedup_vs_fp64_batched"] = value / out["fp64_batched"]["value"]
        out["layer_edep_fp32_vs_fp64_gpu"] = compare_layers(total_and_sigma(layers["fp32"]),
                                                            total_and_sigma(layers["fp64"]))
        from scipy.stats import ks_2samp
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

    # C4 (2^16 mixed e-/e+/gamma, log-uniform 10 MeV - 100 GeV, 4 T) and C5
    # (4096 events of Poisson(100) 10 GeV electrons, scored per event): the
    # FP32-mixed and FP64 batched engines on the same streams, the plain FP64
    # loop (on a bounded sample), per-layer (C5: per-event) agreement;
    # and C3 itself through the CSG volume tree
    extra = {}
    for name, fn in (("c4", lambda: configs.c4(65536)), ("c5", lambda: configs.c5(4096, 100)),
                     ("c3_csg_tree", lambda: configs.c3())):
        c, pr, nv = fn()
        c.first_substream = rank * len(pr[0])
        if name == "c3_csg_tree":
            dm.load_geometry(geometry.calorimeter(axis=c.axis))
            c.geometry = 2
        tens = {k: torch.as_tensor(x, device="cuda") for k, x in zip(("t", "E", "p", "d"), pr[:4])}
        evx = torch.as_tensor(pr[4], device="cuda") if pr[4] is not None else None
        ox = torch.zeros((c.nevents, nv), dtype=torch.float64, device="cuda")
        m32, s32, _, st = timed(1, 1, 1, 1, c=c, tens=tens, events=evx, out=ox)
        e32 = ox.cpu().numpy()
        rec = {"track_steps_per_s": s32 / (m32 / 1e3), "primaries_per_s": len(pr[0]) / (m32 / 1e3),
               "primaries": len(pr[0]), "steps": int(s32), "ms": m32}
        if name == "c5":
            rec["events"] = int(c.nevents)
            rec["events_per_s"] = c.nevents / (m32 / 1e3)
        if name != "c3_csg_tree" and not args.no_fp64:
            # one warm-up run: the first FP64 run of a workload sizes the
            # engine's FP64 stores and captures its graphs
            m64, s64, _, _ = timed(0, 1, 1, 1, c=c, tens=tens, events=evx, out=ox)
            e64 = ox.cpu().numpy()
            rec["fp64_batched"] = {"track_steps_per_s": s64 / (m64 / 1e3), "ms": m64, "steps": int(s64)}
            rec["fp32_over_fp64_batched"] = (s32 / m32) / (s64 / m64)
            # plain FP64 loop on a bounded sample: C4 its first 8192
            # primaries, C5 its first 64 events
            if name == "c5":
                k = int(np.searchsorted(pr[4], 64))
                sub = {kk: v[:k] for kk, v in tens.items()}
                c.nevents = 64
                op = torch.zeros((64, nv), dtype=torch.float64, device="cuda")
                mp, sp, _, _ = timed(0, 0, 1, 0, c=c, tens=sub, events=evx[:k], out=op)
                c.nevents = 4096
                rec["fp64_plain"] = {"track_steps_per_s": sp / (mp / 1e3), "ms": mp, "steps": int(sp),
                                     "sample": "events 0-63 (%d primaries)" % k}
            else:
                sub = {kk: v[:8192] for kk, v in tens.items()}
                mp, sp, _, _ = timed(0, 0, 1, 0, c=c, tens=sub, out=ox)
                rec["fp64_plain"] = {"track_steps_per_s": sp / (mp / 1e3), "ms": mp, "steps": int(sp),
                                     "sample": "primaries 0-8191"}
            rec["fp32_over_fp64_plain"] = (s32 / m32) / (rec["fp64_plain"]["track_steps_per_s"] / 1e3)
            l32, l64 = layer_sums(e32).sum(0), layer_sums(e64).sum(0)
            big = l64 > 0.002 * l64.sum()
            rel = np.abs(l32 - l64)[big] / l64[big]
            rec["layer_edep_fp32_vs_fp64_gpu"] = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                                                  "total_rel": float(abs(l32.sum() - l64.sum()) / l64.sum()),
                                                  "layers_compared": int(big.sum())}
            if name == "c5":
                # per event: the largest relative difference over the layers
                # holding > 2% of that event's deposit, then max and mean over events
                a32, a64 = layer_sums(e32), layer_sums(e64)
                tot = a64.sum(1, keepdims=True)
                mask = a64 > 0.02 * tot
                r = np.where(mask, np.abs(a32 - a64) / np.where(mask, a64, 1.0), 0.0).max(1)
                rec["event_layer_edep_fp32_vs_fp64_gpu"] = {
                    "max_over_events": float(r.max()), "mean_over_events": float(r.mean()),
                    "median_over_events": float(np.median(r)), "layers": "> 2% of the event's deposit",
                    "event_total_rel_max": float((np.abs(a32.sum(1) - a64.sum(1)) / a64.sum(1)).max())}
        if name == "c4" and not args.no_tune_c4:
            # the launch-setting sweep on a quarter of C4 (one run per
            # setting), then the whole of C4 at the winner (untimed sweep)
            c.precision, c.engine, c.profile = 1, 1, 0
            nt = 16384
            trials = gx.autotune(dm, c, tens["t"][:nt], tens["E"][:nt], tens["p"][:nt], tens["d"][:nt], nvol=nv,
                                 repeats=1)
            mt, stt, _, _ = timed(1, 1, 1, 1, c=c, tens=tens, events=evx, out=ox)
            rec["autotuned"] = {"track_steps_per_s": stt / (mt / 1e3), "primaries_per_s": len(pr[0]) / (mt / 1e3),
                                "ms": mt, "steps": int(stt), "over_default": (stt / mt) / (s32 / m32),
                                "setting": dict({k: trials[0][k] for k in LAUNCH_KEYS},
                                                fetch_min_gamma=trials[0]["fetch_min_gamma"]),
                                "trials": len(trials),
                                "tuned_on": "primaries 0-%d, one run per setting" % (nt - 1)}
            for k in LAUNCH_KEYS:
                setattr(c, k, 0)
            c.fetch_min_by_type[0] = 0
        extra[name] = rec
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
    k_ms = stp["transport_ms"][k]
    k_steps = stp["transport_steps"][k]
    k_records = stp["transport_read"][k] + stp["transport_written"][k]
    # algorithmic bytes: one read and one write of the track record per step
    # (a step reads and writes the state once); the kernel keeps a track in
    # registers across steps, so the records it actually moves are fewer
    nbytes = k_steps * 2 * stp["bytes_per_track"]
    moved = k_records * stp["bytes_per_track"]
    achieved = nbytes / (k_ms / 1e3) / 1e9
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
            traffic = per[k] * k_records / launches_k
    pipes = None
    pf = os.path.join(REPO, "profiles", "transport_kernel_pipes.txt")
    if os.path.exists(pf):
        # FP64 / FP32 / ALU pipe and issue utilisation (% of peak) of this
        # kernel from the same ncu capture: the kernel is latency-bound
        for line in open(pf):
            f = line.split()
            if len(f) >= 6 and not line.startswith("#") and int(f[0]) == k:
                pipes = {"fp64_pct": float(f[1]), "fp32_fma_pct": float(f[2]), "alu_pct": float(f[3]),
                         "issue_pct": float(f[4]), "active_lanes_of_32": float(f[5]), "source": "ncu"}
                if len(f) >= 8:  # the same kernel on launches of the full batch
                    pipes["active_lanes_of_32_full_size"] = float(f[6])
                    pipes["issue_pct_full_size"] = float(f[7])
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "traffic": traffic,
                       "kernel": "k_transport<float,%d,0> (%s)" % (k, ["gamma", "e-", "e+"][k]),
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                       "algorithmic_bytes_per_launch": nbytes / launches_k,
                       "steps_per_launch": k_steps / launches_k,
                       "record_bytes_moved_per_launch": moved / launches_k,
                       "record_bytes_moved_gbs": moved / (k_ms / 1e3) / 1e9,
                       "avg_launch_ms": k_ms / launches_k,
                       "share_of_step_kernel_time": k_ms / max(1e-9, sum(stp["step_ms"])),
                       "records_per_launch": k_records / launches_k,
                       "pipes": pipes}

    if rank == 0 and not args.no_cpu:
        nth = os.cpu_count() or 1
        # the CPU baseline at equal statistics: the oracle (pinned to the
        # reference's own code) on the whole C3 batch of this rank, all host
        # cores, scored in the same ten sub-batches
        orc, flags = load_oracle()
        t0 = time.perf_counter()
        r = orc.transport(c3_oracle_config(nth, NSUB, cfg.first_substream), types, E, pos, d, events=ev_np,
                          nvol=nvol, nevents=NSUB)
        dtc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": r["steps"] / dtc, "unit": UNIT, "cores": nth, "kind": "port",
                               "sample": "the whole C3 batch (%d primaries, %d track-steps), oracle step loop, %s, "
                                         "%d threads, %.1f s" % (nprim, r["steps"], flags, nth, dtc)}
        lo = layer_sums(r["edep"])
        out["layer_edep_fp32_vs_oracle"] = compare_layers(total_and_sigma(layers["fp32"]), total_and_sigma(lo))
        if "fp64" in layers:
            out["layer_edep_fp64_gpu_vs_oracle"] = compare_layers(total_and_sigma(layers["fp64"]),
                                                                  total_and_sigma(lo))
        from scipy.stats import ks_2samp
        ks = ks_2samp(p32, r["primary_steps"])
        out["primary_step_count_ks_fp32_vs_oracle"] = {"statistic": float(ks.statistic), "pvalue": float(ks.pvalue),
                                                       "mean_oracle": float(r["primary_steps"].mean())}
        # the FP64 parity variant against the oracle's parity build, whole batch
        if "fp64_parity" in layers:
            og, _ = load_oracle(parity=True)
            t0 = time.perf_counter()
            rg = og.transport(c3_oracle_config(nth, NSUB, cfg.first_substream), types, E, pos, d, events=ev_np,
                              nvol=nvol, nevents=NSUB)
            lg = layer_sums(rg["edep"]).sum(0)
            lp = layers["fp64_parity"].sum(0)
            out["fp64_parity_vs_oracle_parity_build"] = {
                "primaries": nprim, "same_step_count": int(np.sum(ppar == rg["primary_steps"])),
                "steps_gpu": int(ppar.sum()), "steps_oracle": int(rg["primary_steps"].sum()),
                "layer_edep_max_rel": float((np.abs(lp - lg) / np.maximum(lg, 1e-300))[lg > 0].max()),
                "oracle_seconds": time.perf_counter() - t0}
        # bounded CPU samples of C4 and C5 on all host cores
        from oracle_ctypes import oracle_config
        for name in ("c4", "c5"):
            if name == "c4":
                c, pr, nv = configs.c4(65536)
                n, t_used = 64, 0.0
                while True:
                    t0 = time.perf_counter()
                    rr = orc.transport(oracle_config(c, nth), *[x[:n] for x in pr[:4]], nvol=nv)
                    t_used = time.perf_counter() - t0
                    if t_used >= 0.5 * args.cpu_seconds or n >= 65536:
                        break
                    n = int(min(65536, max(2 * n, n * args.cpu_seconds * 0.7 / max(t_used, 1e-3))))
                extra["c4"]["cpu_baseline"] = {"track_steps_per_s": rr["steps"] / t_used,
                                               "primaries_per_s": n / t_used, "cores": nth, "kind": "port",
                                               "sample": "the first %d of the 65536 C4 primaries, %.1f s" % (n, t_used)}
            else:
                c, pr, nv = configs.c5(4096, 100)
                ne, t_used = 2, 0.0
                while True:
                    k = int(np.searchsorted(pr[4], ne))
                    c.nevents = ne
                    t0 = time.perf_counter()
                    rr = orc.transport(oracle_config(c, nth), *[x[:k] for x in pr[:4]], events=pr[4][:k], nvol=nv,
                                       nevents=ne)
                    t_used = time.perf_counter() - t0
                    if t_used >= 0.5 * args.cpu_seconds or ne >= 4096:
                        break
                    ne = int(min(4096, max(2 * ne, ne * args.cpu_seconds * 0.7 / max(t_used, 1e-3))))
                extra["c5"]["cpu_baseline"] = {"track_steps_per_s": rr["steps"] / t_used, "events_per_s": ne / t_used,
                                               "cores": nth, "kind": "port",
                                               "sample": "events 0-%d of the 4096 C5 events (%d primaries), %.1f s"
                                                         % (ne - 1, k, t_used)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    dm.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
