"""CUDA kernels, called through the C ABI, against the golden vectors of the
reference's own code and against the oracle (FP64).

Tolerances: MRG32k3a draws and stream states are compared bit for bit; table
lookups, interaction outputs, step limits and the helix to 1e-12 relative
(the kernels evaluate the same formulas, with fused multiply-adds and CUDA's
FP64 math library instead of glibc's)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as g
    return g.ProxyDataManager()


def close(a, b, rtol=RTOL, scale=None):
    """|a - b| <= rtol * scale elementwise (scale defaults to |b|); NaNs must coincide."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape
    s = np.abs(b) if scale is None else np.broadcast_to(np.asarray(scale, dtype=np.float64), b.shape)
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    assert np.array_equal(nan_a, nan_b)
    ok = ~nan_b
    a, b, s = a[ok], b[ok], s[ok]
    diff = np.abs(a - b)
    bad = (diff > rtol * np.maximum(s, 1e-300)) & (a != b)
    assert not bad.any(), ("%d of %d beyond rtol %g; worst |a-b|/scale = %.3g" %
                           (bad.sum(), bad.size, rtol, (diff / np.maximum(s, 1e-300)).max()),
                           np.nonzero(bad)[0][:5], a[bad][:5], b[bad][:5])


# ------------------------------------------------------------------ MRG32k3a
def test_rng_first_1000_draws_bit_exact(golden):
    from geantexascalepilot_b200 import MRG32k3a
    g = golden["mrg"]
    st = MRG32k3a.from_states(g["seed"])
    out = MRG32k3a.uniform(st, 1000).cpu().numpy()[:, 0]
    assert np.array_equal(out, g["draws"])
    assert np.array_equal(MRG32k3a.to_states(st).numpy()[0], g["state_after"])


@pytest.mark.parametrize("seed", [12345, 2024, 7])
def test_rng_substreams_device_skip_ahead(golden, seed):
    from geantexascalepilot_b200 import MRG32k3a
    want = golden["mrg"]["substreams_%d" % seed]
    st = MRG32k3a.substreams([seed] * 6, 0, want.shape[0])
    assert np.array_equal(MRG32k3a.to_states(st).numpy(), want)
    st5 = MRG32k3a.substreams([seed] * 6, 5, 1)
    assert np.array_equal(MRG32k3a.to_states(st5).numpy()[0], want[5])


def test_rng_advance_and_stream_id(golden):
    from geantexascalepilot_b200 import MRG32k3a
    g = golden["mrg"]
    for (e, c), want in zip(g["adv_cases"], g["adv"]):
        st = MRG32k3a.from_states(g["seed"])
        MRG32k3a.advance(st, int(e), int(c))
        assert np.array_equal(MRG32k3a.to_states(st).numpy()[0], want), (e, c)
    st = MRG32k3a.stream_id(range(4))
    out = MRG32k3a.uniform(st, 4).cpu().numpy()
    assert np.array_equal(out.T, g["stream_id_draws"])


def test_rng_many_streams_vs_oracle(oracle):
    from geantexascalepilot_b200 import MRG32k3a
    first = (1 << 40) + 12345
    st = MRG32k3a.substreams([2024.0] * 6, first, 4096)
    ref = oracle.substreams(np.full(6, 2024.0), first, 4096)
    assert np.array_equal(MRG32k3a.to_states(st).numpy(), ref)
    draws = MRG32k3a.uniform(st, 257).cpu().numpy()
    ref_draws, ref_st = oracle.mrg_draws(ref, 257)
    assert np.array_equal(draws, ref_draws)
    assert np.array_equal(MRG32k3a.to_states(st).numpy(), ref_st)


# ------------------------------------------------------------------- tables
def test_tables_vs_golden(dm, golden):
    g = golden["tables"]
    for t in range(20):
        if t in (4, 5):
            continue
        for m in range(3):
            got = dm.table_value(t, m, g["E"]).cpu().numpy()
            close(got, g["values"][t, m], rtol=1e-13)


def test_inverse_range_vs_golden(dm, golden):
    g = golden["tables"]
    for k, t in enumerate((4, 5)):
        for m in range(3):
            close(dm.inv_range_value(t, m, g["R"]).cpu().numpy(), g["invrange"][k, m], rtol=1e-13)


def test_sb_2d_and_cuts_vs_golden(dm, golden):
    g = golden["tables"]
    for which in range(3):
        close(dm.sb_value(which, g["sb_x"], g["sb_y"]).cpu().numpy(), g["sb_values"][which], rtol=1e-14)
    got = np.array([[dm.GetCutValue(i, p) for p in range(3)] for i in range(3)])
    assert np.array_equal(got, g["cuts"])


# ------------------------------------------------------------------- models
MODELS = {"kn": "ProxyKleinNishina", "sg": "ProxySauterGavrila", "bh": "ProxyBetheHeitler",
          "sb": "ProxySeltzerBerger", "mb": "ProxyMollerScattering"}


def _dir_tolerance(out_dir, in_dir):
    """Allowed deviation of a sampled direction: 1e-12, plus the conditioning of
    the reference's sin(theta) = sqrt((1 - cos)(1 + cos)) near cos -> 1, where
    one ulp of cos (CUDA vs glibc transcendental functions) moves sin(theta)
    by ~1e-16 / sin(theta)."""
    c = np.clip(np.einsum("...k,...k->...", out_dir, in_dir), -1.0, 1.0)
    return 1e-12 + 1e-14 / np.sqrt(np.maximum(1.0 - np.abs(c), 1e-30))


def _check_inter(got, want_get, dir_in, rtol=RTOL):
    for key in ("E", "edep", "sec_E"):
        w = want_get(key)
        scale = None if key == "E" else np.maximum(np.abs(w), 1e-30)
        close(got[key].cpu().numpy(), w, rtol=rtol, scale=scale)
    w = want_get("dir")
    close(got["dir"].cpu().numpy(), w, rtol=1.0, scale=_dir_tolerance(w, dir_in)[:, None])
    w = want_get("sec_dir")
    close(got["sec_dir"].cpu().numpy(), w, rtol=1.0, scale=_dir_tolerance(w, dir_in[:, None, :])[..., None])
    for key in ("status", "nsec", "sec_type"):
        assert np.array_equal(got[key].cpu().numpy(), want_get(key)), key


@pytest.mark.parametrize("model", list(MODELS))
def test_models_quirk_mode_vs_reference_golden(dm, golden, model):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import MRG32k3a
    g = golden["models_quirk"]
    m = getattr(gx, MODELS[model])(dm, mode=gx.MODE_QUIRK, Z=10, sb_table=0)
    st = MRG32k3a.from_states(g[model + "_states"])
    out = m.SampleSecondaries(g[model + "_E_in"], g[model + "_dir_in"], st)
    _check_inter(out, lambda k: g[model + "_" + k], g[model + "_dir_in"])
    assert np.array_equal(MRG32k3a.to_states(st).numpy(), g[model + "_states_out"])


PHYS = [("kn", 82, 0.0, 1e-4, 1e5), ("sg", 82, 0.0, 1e-4, 1e2), ("sg", 18, 0.0, 1e-4, 1e2), ("bh", 82, 0.0, 1.03, 1e5),
        ("bh", 18, 0.0, 1.03, 1e5), ("sb", 82, 0.0945861383106, 0.2, 1e5), ("sb", 18, 0.00520596294409, 0.01, 1e5),
        ("mb", 82, 1.00386448578, 2.1, 1e5), ("mb", 18, 0.272576829155, 0.6, 1e5),
        ("bhabha", 82, 1.00386448578, 1.1, 1e5), ("annih", 82, 0.0, 1e-3, 1e5)]


@pytest.mark.parametrize("model,Z,cut,lo,hi", PHYS)
def test_models_physics_mode_vs_oracle(dm, oracle, model, Z, cut, lo, hi):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import MRG32k3a
    rng = np.random.default_rng(Z * 7 + len(model))
    n = 4096
    E = 10 ** rng.uniform(np.log10(lo), np.log10(hi), n)
    if model == "annih":
        E[:64] = 0.0  # at rest
    D = rng.normal(size=(n, 3))
    D /= np.linalg.norm(D, axis=1)[:, None]
    D[:3] = [[0, 0, 1], [0, 0, -1], [1, 0, 0]]
    states = oracle.substreams(np.full(6, 7.0), 1000 + Z, n)
    dfac = {82: 1.4281e-8, 18: 2.9e-9}[Z] if model == "sb" else 0.0
    sbt = {82: 2, 18: 1}[Z]
    ids = {"kn": gx.KLEIN_NISHINA, "sg": gx.SAUTER_GAVRILA, "bh": gx.BETHE_HEITLER, "sb": gx.SELTZER_BERGER,
           "mb": gx.MOLLER, "bhabha": gx.BHABHA, "annih": gx.ANNIHILATION}
    m = gx.api._Model(dm, mode=gx.MODE_PHYSICS, Z=Z, cut=cut, density_factor=dfac, sb_table=sbt)
    m.model_id = ids[model]
    st = MRG32k3a.from_states(states)
    got = m.SampleSecondaries(E, D, st)
    p = oracle.params(mode=1, Z=Z, cut=cut, density_factor=dfac, sb={82: "pb", 18: "ar"}[Z])
    want = oracle.interact(model, states, E, D, p)
    _check_inter(got, lambda k: want[k], D, rtol=1e-11)
    assert np.array_equal(MRG32k3a.to_states(st).numpy(), want["states"])


def test_cross_sections_vs_golden(golden):
    import geantexascalepilot_b200 as gx
    g = golden["xs"]
    kn = gx.ProxyKleinNishina(None)
    mb = gx.ProxyMollerScattering(None)
    for i, z in enumerate(g["Z"]):
        close(kn.CrossSectionPerAtom(z, g["E"]).cpu().numpy(), g["kn"][i], rtol=1e-13)
        close(mb.CrossSectionPerAtom(z, g["E"]).cpu().numpy(), g["mb"][i], rtol=1e-13)


# ---------------------------------------------------------------- processes
def test_post_step_gpil_vs_golden(dm, golden):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import MRG32k3a
    g = golden["processes"]
    procs = [gx.ProxyCompton(dm), gx.ProxyConversion(dm), gx.ProxyPhotoElectric(dm), gx.ProxyBremsstrahlung(dm),
             gx.ProxyIonization(dm)]
    for p in range(5):
        sel = np.nonzero(g["gpil_proc"] == p)[0]
        st = MRG32k3a.from_states(g["gpil_states"][sel])
        nil = torch.tensor(g["gpil_nil"][sel], device="cuda")
        saved = torch.tensor(g["gpil_saved"][sel], device="cuda")
        step = procs[p].PostStepGPIL(g["gpil_E"][sel], g["gpil_pstep"][sel], nil, saved, st, mat=2)
        close(step.cpu().numpy(), g["gpil_step"][sel], rtol=1e-13)
        close(nil.cpu().numpy(), g["gpil_nil_out"][sel], rtol=1e-13)
        close(saved.cpu().numpy(), g["gpil_saved_out"][sel], rtol=1e-13)
        assert np.array_equal(MRG32k3a.to_states(st).numpy(), g["gpil_states_out"][sel])


def test_ionisation_along_step_vs_golden(dm, golden):
    import geantexascalepilot_b200 as gx
    g = golden["processes"]
    ion = gx.ProxyIonization(dm)
    close(ion.AlongStepGPIL(g["agpil_mat"], g["agpil_E"]).cpu().numpy(), g["agpil_step"], rtol=1e-12)
    d = g["adoit_defined"]
    E, edep = ion.AlongStepDoIt(g["adoit_mat"][d], g["adoit_step"][d], g["adoit_E"][d])
    close(E.cpu().numpy(), g["adoit_E_out"][d], rtol=1e-11, scale=g["adoit_E"][d])
    close(edep.cpu().numpy(), g["adoit_edep"][d], rtol=1e-11, scale=g["adoit_E"][d])


def test_ionisation_physics_mode_vs_oracle(dm, oracle):
    import geantexascalepilot_b200 as gx
    rng = np.random.default_rng(5)
    ion = gx.ProxyIonization(dm)
    for charge in (-1, 1):
        mat = 1 + np.arange(2000) % 2
        E = 10 ** rng.uniform(-4.5, 5, 2000)
        got = ion.AlongStepGPIL(mat, E, mode=gx.MODE_PHYSICS, charge=charge).cpu().numpy()
        want = [oracle.ioni_along_gpil(1, charge, int(m), e) for m, e in zip(mat, E)]
        close(got, want, rtol=1e-12)
        rg = oracle.table_value(19 if charge > 0 else 18, 1, E)
        step = rg * rng.choice([0.001, 0.05, 0.3, 0.9, 1.2], 2000)
        Eo, ed = ion.AlongStepDoIt(mat, step, E, mode=gx.MODE_PHYSICS, charge=charge)
        want = np.array([oracle.ioni_along_doit(1, charge, int(m), s, e) for m, s, e in zip(mat, step, E)])
        close(Eo.cpu().numpy(), want[:, 0], rtol=1e-10, scale=E)
        close(ed.cpu().numpy(), want[:, 1], rtol=1e-10, scale=E)


def test_helix_vs_golden(golden):
    import geantexascalepilot_b200 as gx
    g = golden["helix"]
    h = gx.ConstFieldHelixStepper(g["B"])
    npos, ndir = h.DoStepArr(g["pos"], g["dir"], g["charge"], g["mom"], g["step"])
    scale = np.abs(g["pos"]).max() + np.abs(g["step"]).max()
    close(npos.cpu().numpy(), g["newpos"], rtol=1e-12, scale=scale)
    close(ndir.cpu().numpy(), g["newdir"], rtol=1e-12, scale=1.0)


# ------------------------------------------------------------------ edges
def test_empty_batches_and_argument_errors(dm):
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import MRG32k3a, GxError
    st = MRG32k3a.substreams([1.0] * 6, 0, 0)
    assert st.shape == (6, 0)
    assert dm.table_value(8, 1, np.zeros(0)).numel() == 0
    out = gx.ProxyKleinNishina(dm).SampleSecondaries(np.zeros(0), np.zeros((0, 3)), st)
    assert out["E"].numel() == 0
    with pytest.raises(GxError):
        dm.table_value(25, 1, np.ones(3))
    with pytest.raises(GxError):
        MRG32k3a.substreams([5e9] * 6, 0, 4)  # seed word >= m1
