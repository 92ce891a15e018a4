"""Whole transport on the GPU against the oracle's step loop on identical
MRG32k3a streams, the two engines against each other, FP32-mixed against
FP64, energy conservation, and the host-buffer entry point."""
import numpy as np
import pytest
import torch
from oracle_ctypes import oracle_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as g
    return g.ProxyDataManager()


def run_gpu(dm, cfg, prims, nvol, precision=0, engine=1, primary_steps=False, **kw):
    import geantexascalepilot_b200 as g
    cfg.precision = precision
    cfg.engine = engine
    for k, v in kw.items():
        setattr(cfg, k, v)
    types, E, pos, d, ev = prims
    edep, st, ps = g.transport(dm, cfg, types, E, pos, d, events=ev, nvol=nvol, primary_steps=primary_steps)
    torch.cuda.synchronize()
    return edep.cpu().numpy(), st, (ps.cpu().numpy() if ps is not None else None)


def run_oracle(oracle, cfg, prims, nvol):
    types, E, pos, d, ev = prims
    return oracle.transport(oracle_config(cfg), types, E, pos, d, events=ev, nvol=nvol, nevents=cfg.nevents)


def test_c1_gamma_box_matches_oracle_track_by_track(dm, oracle):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c1(4000)
    edep, st, ps = run_gpu(dm, cfg, prims, nvol, primary_steps=True)
    ref = run_oracle(oracle, cfg, prims, nvol)
    same = np.mean(ps == ref["primary_steps"])
    assert same >= 0.999, same
    assert st["steps"] == ref["steps"] or abs(st["steps"] - ref["steps"]) <= 3
    assert abs(st["n_pair"] - ref["n_pair"]) <= 2
    assert np.isclose(edep.sum(), ref["edep"].sum(), rtol=1e-6)
    assert np.isclose(st["escaped"], ref["escaped"], rtol=1e-5)


def test_showers_fp64_match_oracle_no_field(dm, oracle):
    """Without a field the FP64 engine and the oracle follow the same tracks."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(16)
    edep, st, _ = run_gpu(dm, cfg, prims, nvol)
    ref = run_oracle(oracle, cfg, prims, nvol)
    assert st["errors"] == 0
    assert abs(st["steps"] - ref["steps"]) <= 1e-5 * ref["steps"]
    assert abs(st["tracks"] - ref["tracks"]) <= 1e-4 * ref["tracks"]
    np.testing.assert_allclose(edep.ravel(), ref["edep"].ravel(), rtol=1e-6, atol=1e-6 * ref["edep"].max())


NSUB = 10


def layer_totals(edep_events):
    """[NSUB, 100] slab tallies of NSUB sub-batches -> per-layer totals and
    their standard deviations (sqrt(NSUB) x the sub-batches' spread)."""
    per = np.asarray(edep_events).reshape(NSUB, -1, 2).sum(2)
    return per.sum(0), np.sqrt(NSUB * per.var(0, ddof=1))


def assert_shower_bar(a, b):
    """The bar of the C3 comparisons: every layer holding more than 0.2% of
    the deposit within 0.5% and within 3 standard deviations."""
    (ta, sa), (tb, sb) = a, b
    big = tb > 0.002 * tb.sum()
    rel = np.abs(ta - tb)[big] / tb[big]
    pull = np.abs(ta - tb)[big] / np.sqrt(sa[big] ** 2 + sb[big] ** 2)
    assert rel.max() <= 0.005, rel.max()
    assert pull.max() <= 3.0, pull.max()


def c3_sub_batches(n_e, n_g):
    """C3 with primary i scored as event i % NSUB (sub-batches of one mix)."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(n_e, n_g)
    ev = (np.arange(n_e + n_g) % NSUB).astype(np.int32)
    cfg.nevents = NSUB
    return cfg, prims[:4] + (ev,), nvol


def test_showers_fp64_match_oracle_in_field(dm, oracle):
    """The FP64 engine (with contraction and CUDA's functions) against the
    oracle on the same streams in 4 T: tracks part at the last bits, so
    statistically -- 2000 showers in ten sub-batches, every layer within 0.5%
    and 3 standard deviations.  (The FP64 parity variant agrees track by track:
    test_gpu_parity_transport.py.)"""
    cfg, prims, nvol = c3_sub_batches(1000, 1000)
    edep, st, _ = run_gpu(dm, cfg, prims, nvol)
    ref = run_oracle(oracle, cfg, prims, nvol)
    assert st["errors"] == 0
    assert abs(st["steps"] - ref["steps"]) <= 2e-3 * ref["steps"]
    assert_shower_bar(layer_totals(edep), layer_totals(ref["edep"]))


def test_energy_conservation(dm):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(16, 16)
    for prec, tol in ((0, 1e-9), (1, 1e-5)):
        edep, st, _ = run_gpu(dm, cfg, prims, nvol, precision=prec)
        e0 = prims[1].sum()
        assert abs(edep.sum() + st["escaped"] - e0) <= tol * e0, (prec, edep.sum(), st["escaped"], e0)


def test_plain_and_batched_engines_agree(dm):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(8)
    a, sa, _ = run_gpu(dm, cfg, prims, nvol, engine=0)
    b, sb, _ = run_gpu(dm, cfg, prims, nvol, engine=1)
    assert sa["steps"] == sb["steps"] and sa["tracks"] == sb["tracks"]
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * a.max())


def test_fp32_mixed_vs_fp64_and_oracle_per_layer(dm, oracle):
    """The bar of the FP32-mixed engine at C3 (10 GeV e- and gamma, 4 T): per
    layer within 0.5% and 3 standard deviations of the FP64 engine on the same
    streams and of the CPU oracle -- 2000 showers in ten sub-batches."""
    cfg, prims, nvol = c3_sub_batches(1000, 1000)
    e32, s32, _ = run_gpu(dm, cfg, prims, nvol, precision=1)
    e64, _, _ = run_gpu(dm, cfg, prims, nvol, precision=0)
    ref = run_oracle(oracle, cfg, prims, nvol)
    assert s32["errors"] == 0
    assert_shower_bar(layer_totals(e32), layer_totals(e64))
    assert_shower_bar(layer_totals(e32), layer_totals(ref["edep"]))


def test_host_entry_point_equals_device_path(dm):
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(4)
    a, sa, _ = run_gpu(dm, cfg, prims, nvol)
    types, E, pos, d, ev = prims
    b, sb = g.transport_host(dm, cfg, types, E, pos, d, nvol=nvol)
    assert sa["steps"] == sb["steps"]
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * a.max())


def test_per_event_tallies_match_oracle(dm, oracle):
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c5(nevents=12, mean=2)
    prims = (prims[0], np.full(len(prims[0]), 500.0), prims[2], prims[3], prims[4])
    edep, st, _ = run_gpu(dm, cfg, prims, nvol)
    ref = run_oracle(oracle, cfg, prims, nvol)
    assert edep.shape == (12, nvol)
    np.testing.assert_allclose(edep.sum(1), ref["edep"].sum(1), rtol=1e-6)


def test_shards_on_global_substreams_sum_to_the_whole(dm):
    """Three contiguous shards run one after another (as three GPUs would run
    them), each on the substreams of its global primary indices: the summed
    tallies and counters equal one run over all primaries."""
    from geantexascalepilot_b200 import configs, sharding
    cfg, prims, nvol = configs.c3(6, 6)
    whole, sw, _ = run_gpu(dm, cfg, prims, nvol)
    tot = np.zeros_like(whole)
    steps = tracks = 0
    for r in range(3):
        sub, first = sharding.shard(prims, r, 3)
        cfg.first_substream = first
        e, st, _ = run_gpu(dm, cfg, sub, nvol)
        tot += e
        steps += st["steps"]
        tracks += st["tracks"]
    cfg.first_substream = 0
    assert steps == sw["steps"] and tracks == sw["tracks"]
    np.testing.assert_allclose(tot, whole, rtol=1e-9, atol=1e-9 * whole.max())


def test_autotune_and_launch_settings_leave_results_unchanged(dm):
    """The sweep returns its trials and writes the winner into the config; any
    launch setting transports the same tracks (per-primary substreams)."""
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(6, 6)
    e0, s0, ps0 = run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True)
    trials = g.autotune(dm, cfg, *prims[:4], nvol=nvol, repeats=1)
    assert len(trials) >= 30
    # the sweep spans 64- to 1024-thread blocks and the compaction interval
    assert {t["block_size"] for t in trials} == {64, 128, 256, 512, 1024}
    assert {t["interaction_interval"] for t in trials} >= {1, 2, 4, 8}
    assert {t["fetch_min_gamma"] for t in trials} >= {1, 8, 16, 24}
    best = trials[0]
    assert best["steps_per_ms"] == max(t["steps_per_ms"] for t in trials) > 0
    assert (cfg.block_size, cfg.blocks_per_sm, cfg.graph_iters, cfg.interaction_interval) == (
        best["block_size"], best["blocks_per_sm"], best["graph_iters"], best["interaction_interval"])
    assert cfg.fetch_min_by_type[0] == best["fetch_min_gamma"]
    assert cfg.block_size in (64, 128, 256, 512, 1024) and cfg.blocks_per_sm in (1, 2, 4, 5, 6, 8)
    e1, s1, ps1 = run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True)
    assert s1["steps"] == s0["steps"] and s1["tracks"] == s0["tracks"]
    assert np.array_equal(ps0, ps1)
    np.testing.assert_allclose(e1, e0, rtol=1e-5, atol=1e-6 * e0.max())
    for k in ("block_size", "blocks_per_sm", "steps_per_launch", "graph_iters", "refill_below", "wave_energy",
              "interaction_interval"):
        setattr(cfg, k, 0)
    cfg.fetch_min_by_type[0] = 0


@pytest.mark.parametrize("precision", [0, 1])
def test_wide_blocks_and_compaction_interval_leave_results_unchanged(dm, precision):
    """512- and 1024-thread blocks (the variants held to 64 registers) and
    interaction kernels run every 3rd or 4th iteration (interacting tracks
    wait in their buffers) transport the same tracks as the defaults."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(12, 12)
    ref = run_gpu(dm, cfg, prims, nvol, precision=precision, primary_steps=True)
    runs = [run_gpu(dm, cfg, prims, nvol, precision=precision, primary_steps=True, block_size=b, blocks_per_sm=bp,
                    interaction_interval=k) for b, bp, k in ((512, 2, 0), (1024, 1, 0), (128, 4, 3), (1024, 2, 4))]
    cfg.block_size, cfg.blocks_per_sm, cfg.interaction_interval = 0, 0, 0
    # FP64 to rounding of the sums; FP32-mixed to float rounding (the wide
    # variants are compiled apart, their float operations may contract differently)
    tol = 1e-9 if precision == 0 else 1e-5
    for e, st, ps in runs:
        assert st["errors"] == 0
        assert st["steps"] == ref[1]["steps"] and st["tracks"] == ref[1]["tracks"]
        assert np.array_equal(ps, ref[2])
        np.testing.assert_allclose(e, ref[0], rtol=tol, atol=tol * ref[0].max())
    assert runs[2][1]["iterations"] >= ref[1]["iterations"]


def test_steps_per_launch_leaves_results_unchanged(dm):
    """One step per transport launch (a track goes back to memory after every
    step) and many steps per launch (it stays in registers) transport the same
    tracks."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(8, 8)
    runs = [run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True, steps_per_launch=k) for k in (1, 7, 4096)]
    cfg.steps_per_launch = 0
    for e, st, ps in runs[1:]:
        assert st["steps"] == runs[0][1]["steps"] and st["tracks"] == runs[0][1]["tracks"]
        assert np.array_equal(ps, runs[0][2])
        np.testing.assert_allclose(e, runs[0][0], rtol=1e-5, atol=1e-6 * runs[0][0].max())
    assert runs[2][1]["iterations"] < runs[0][1]["iterations"]


@pytest.mark.parametrize("precision", [0, 1])
def test_fetch_threshold_leaves_results_unchanged(dm, precision):
    """Warps of the transport kernels that take new records only once many of
    their lanes are idle (up to all 32) transport the same tracks as warps that
    refill every idle lane at once; out-of-range thresholds are refused."""
    import geantexascalepilot_b200 as g
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(8, 8)
    runs = []
    for fm in ((1, 1, 1), (0, 0, 0), (32, 32, 32), (7, 5, 3)):
        for q in range(3):
            cfg.fetch_min_by_type[q] = fm[q]
        runs.append(run_gpu(dm, cfg, prims, nvol, precision=precision, primary_steps=True))
    for e, st, ps in runs[1:]:
        assert st["steps"] == runs[0][1]["steps"] and st["tracks"] == runs[0][1]["tracks"]
        assert np.array_equal(ps, runs[0][2])
        np.testing.assert_allclose(e, runs[0][0], rtol=1e-9, atol=1e-9 * runs[0][0].max())
    for bad in (33, -1):
        cfg.fetch_min_by_type[1] = bad
        with pytest.raises(g.GxError):
            run_gpu(dm, cfg, prims, nvol, precision=precision)
    for q in range(3):
        cfg.fetch_min_by_type[q] = 0


@pytest.mark.parametrize("profile", [0, 1])
def test_record_counters_are_consistent(dm, profile):
    """The record statistics of the batched engine, counted in three places
    (the transport kernels per warp, k_finish from the interaction buffers'
    counters, the interaction kernels per lane): every record a transport
    kernel queued is read once by an interaction kernel, a transport kernel
    writes no more records than it read, and its steps are the run's steps;
    with the graph (profile 0) and without it (profile 1)."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(40, 40)
    _, st, _ = run_gpu(dm, cfg, prims, nvol, precision=1, profile=profile)
    cfg.profile = 0
    assert st["errors"] == 0
    for q in range(3):
        assert st["transport_queued"][q] <= st["transport_written"][q] <= st["transport_read"][q]
        assert st["tracks_read"][q] - st["transport_read"][q] == st["transport_queued"][q], q
        assert st["tracks_written"][q] >= st["transport_written"][q]
    assert sum(st["transport_steps"]) == st["steps"]
    assert st["transport_read"][0] > 0 and st["transport_read"][1] > 0 and st["transport_queued"][2] > 0


def test_step_count_distributions_fp32_vs_fp64(dm):
    """Two-sample Kolmogorov-Smirnov test on the primaries' step counts,
    FP32-mixed against FP64 on the same streams."""
    from scipy.stats import ks_2samp
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(100, 100)
    _, _, p64 = run_gpu(dm, cfg, prims, nvol, precision=0, primary_steps=True)
    _, _, p32 = run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True)
    assert ks_2samp(p32, p64).pvalue > 0.01


def test_small_capacity_uses_the_overflow_stack(dm):
    """A store far smaller than the shower forces deferral to the stack and
    re-injection; the result must not change."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(4)
    a, sa, _ = run_gpu(dm, cfg, prims, nvol, capacity=0)
    b, sb, _ = run_gpu(dm, cfg, prims, nvol, capacity=512, refill_below=64)
    assert sb["errors"] == 0
    assert sa["steps"] == sb["steps"]
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * a.max())


@pytest.mark.parametrize("n,capacity,wave", [(256, 1 << 15, 0.0), (64, 0, 2.0e4)])
def test_injection_by_live_energy_leaves_results_unchanged(dm, n, capacity, wave):
    """C4-like primaries (10 MeV-100 GeV, e-/e+/gamma) through stores far
    smaller than all their showers at once (2^15 slots per type against a
    ~2.8 TeV total), or with a live-energy bound below single primaries'
    energies (20 GeV, so each such primary waits until nothing is in flight):
    the run completes without overflow and every track takes the same steps as
    with all primaries injected at once."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c4(n)
    a, sa, pa = run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True)
    b, sb, pb = run_gpu(dm, cfg, prims, nvol, precision=1, primary_steps=True, capacity=capacity, wave_energy=wave)
    cfg.capacity, cfg.wave_energy = 0, 0.0
    assert sa["errors"] == 0 and sb["errors"] == 0
    assert sb["iterations"] > sa["iterations"]
    assert sa["steps"] == sb["steps"] and sa["tracks"] == sb["tracks"]
    assert np.array_equal(pa, pb)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * a.max())
    # primary positrons bring their rest energy (deposited or escaping with them)
    e0 = prims[1].sum() + 2 * 0.510998910 * np.count_nonzero(prims[0] == 2)
    assert abs(b.sum() + sb["escaped"] - e0) <= 1e-5 * e0


def test_mixed_primaries_conserve_energy_and_agree_fp32_fp64(dm):
    """C4's mixed e-/e+/gamma primaries (10 MeV - 100 GeV): every primary
    positron's rest energy ends up deposited or escaping (annihilation, or
    leaving with its 2 m_e), so deposits + escaped = kinetic energies +
    2 m_e per primary positron, to FP64 rounding; FP32-mixed agrees per layer."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c4(96)
    e0 = prims[1].sum() + 2 * 0.510998910 * np.count_nonzero(prims[0] == 2)
    out = {}
    for prec, tol in ((0, 1e-9), (1, 1e-5)):
        e, st, _ = run_gpu(dm, cfg, prims, nvol, precision=prec)
        assert st["errors"] == 0
        assert abs(e.sum() + st["escaped"] - e0) <= tol * e0, (prec, e.sum() + st["escaped"], e0)
        out[prec] = (e.reshape(-1, 2).sum(1), st)
    a, b = out[0][0], out[1][0]
    big = a > 0.01 * a.sum()
    assert np.all(np.abs(a - b)[big] <= 0.02 * a[big] + 1e-3 * a.sum())
    assert abs(out[0][1]["steps"] - out[1][1]["steps"]) <= 0.02 * out[0][1]["steps"]


def test_transport_edge_cases(dm):
    """no primaries; primaries outside the world or leaving it at once; a
    primary whose event index is outside the tally (an argument error, not a
    store overflow)"""
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import GxError, configs
    cfg, prims, nvol = configs.c3(2, 2)
    for engine in (0, 1):
        for prec in (0, 1):
            e, st, _ = run_gpu(dm, cfg, tuple(p[:0] if p is not None else None for p in prims), nvol,
                               precision=prec, engine=engine)
            assert st["steps"] == 0 and st["errors"] == 0 and not e.any()
    types = np.array([1, 0, 2], np.int32)
    E = np.array([1000.0, 500.0, 250.0])
    pos = np.array([[-500.0, 0, 0], [-200.0, 0, 0], [0.0, 300.0, 0]])  # outside; on the front face; outside
    d = np.array([[1.0, 0, 0], [-1.0, 0, 0], [1.0, 0, 0]])               # the second leaves at once
    e, st, _ = run_gpu(dm, cfg, (types, E, pos, d, None), nvol, precision=0, engine=1)
    assert st["steps"] == 0 and not e.any()
    assert st["escaped"] == pytest.approx(1000.0 + 500.0 + 250.0)  # kinetic energies (primaries never entered)
    ev = np.array([0, 5, 0], np.int32)
    pos[:] = [-200.0, 0, 0]
    d[:] = [1.0, 0, 0]
    cfg.nevents = 2
    with pytest.raises(GxError, match="event index"):
        gx.transport(dm, cfg, types, E, pos, d, events=ev, nvol=nvol)
    cfg.nevents = 1


def test_run_command_line(capsys):
    import json
    from geantexascalepilot_b200 import run
    assert run.main(["c1", "--n", "200", "--precision", "0", "--capacity", "65536"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["workload"] == "c1" and out["primaries"] == 200
    assert out["stats"]["steps"] > 200 and out["stats"]["errors"] == 0


@pytest.mark.parametrize("msc", [1, 2])
def test_multiple_scattering_fp64_matches_oracle(dm, oracle, msc):
    """With multiple scattering on (2: with lateral displacement), the FP64
    engine and the oracle run the same model on the same streams.  Its
    sampling takes logs, exponentials and sines whose last bits differ between
    CUDA and glibc, which can flip a rejection and send a track another way:
    compare the showers statistically (C2, 1 GeV e-, 48 showers)."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(48)
    edep, st, _ = run_gpu(dm, cfg, prims, nvol, msc=msc)
    ref = run_oracle(oracle, cfg, prims, nvol)
    cfg.msc = 0
    assert st["errors"] == 0 and ref["errors"] == 0
    assert abs(st["steps"] - ref["steps"]) <= 0.01 * ref["steps"]
    assert abs(st["tracks"] - ref["tracks"]) <= 0.01 * ref["tracks"]
    e0 = prims[1].sum()
    assert abs(edep.sum() + st["escaped"] - e0) <= 1e-9 * e0
    g = edep.reshape(-1, 2).sum(1)
    o = ref["edep"].reshape(-1, 2).sum(1)
    big = o > 0.002 * o.sum()
    assert np.all(np.abs(g - o)[big] <= 5 * 0.25 / np.sqrt(48) * o[big] + 1e-3 * o.sum())


def test_multiple_scattering_fp32_vs_fp64_and_field(dm):
    """FP32-mixed against FP64 with multiple scattering in 4 T (C3), per layer
    within 1% plus statistics; energy conserved in both."""
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c3(40, 40)
    out = {}
    for prec in (0, 1):
        e, st, _ = run_gpu(dm, cfg, prims, nvol, precision=prec, msc=1)
        e0 = prims[1].sum()
        assert st["errors"] == 0
        assert abs(e.sum() + st["escaped"] - e0) <= (1e-9 if prec == 0 else 1e-5) * e0
        out[prec] = (e.reshape(-1, 2).sum(1), st)
    cfg.msc = 0
    a, b = out[0][0], out[1][0]
    big = a > 0.002 * a.sum()
    assert np.all(np.abs(a - b)[big] <= 0.01 * a[big] + 5 * 0.2 / np.sqrt(80) * a[big])
    assert abs(out[0][1]["steps"] - out[1][1]["steps"]) <= 0.02 * out[0][1]["steps"]


def test_run_command_line_geometry_msc_field_map(capsys):
    """The command line's CSG tree, multiple scattering and field-map options
    reach the engine: the same C3 showers through the tree calorimeter, with
    msc, and through the CMS map all conserve energy."""
    import json
    from geantexascalepilot_b200 import run
    outs = {}
    for name, extra in (("layers", []), ("csg", ["--geometry", "csg"]), ("msc", ["--msc", "2"]),
                        ("map", ["--field-map"])):
        assert run.main(["c3", "--electrons", "20", "--photons", "20", "--capacity", "262144"] + extra) == 0
        outs[name] = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert outs["csg"]["geometry"] == "csg" and outs["msc"]["msc"] == 2 and outs["map"]["field_map"] == "cms"
    e0 = 40 * 1e4
    for name, o in outs.items():
        st = o["stats"]
        assert st["errors"] == 0, name
        assert abs(o["edep_total"] + st["escaped"] - e0) <= 1e-5 * e0, name  # FP32-mixed energies
    # the tree calorimeter is the layered one: same streams, steps within 2%
    a, b = outs["layers"]["stats"]["steps"], outs["csg"]["stats"]["steps"]
    assert abs(a - b) < 0.02 * a
    assert outs["msc"]["stats"]["steps"] > a
