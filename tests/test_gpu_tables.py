"""Physics tables and cuts built by the library instead of read from the
Geant4 dumps, on the GPU: the device-built macroscopic cross sections against
the shipped tables (the same models, up to the material definitions) and
against a CPU restatement of the same integrals; the rebuilt context and the
computed cut table running showers."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
ME = 0.510998910


@pytest.fixture(scope="module")
def dm():
    import geantexascalepilot_b200 as gx
    return gx.ProxyDataManager()


def _grid(lo, hi, n=60):
    return np.exp(np.linspace(np.log(lo), np.log(hi), n))


def _nodes(name, mat):
    """node energies and values of a shipped Geant4-format table"""
    import os
    import geantexascalepilot_b200 as gx
    t = open(os.path.join(gx.DATA_DIR, "table", name + ".asc")).read().split()
    i = 1
    for m in range(int(t[0])):
        siz = int(t[i + 4])
        i += 5
        xy = np.array(t[i:i + 2 * siz], dtype=float).reshape(siz, 2)
        i += 2 * siz
        if m == mat:
            return xy[:, 0], xy[:, 1]


@pytest.mark.parametrize("mat", [1, 2])
def test_built_tables_match_shipped(dm, mat):
    """At the shipped tables' own node energies (between nodes the shipped
    spline itself is off by up to 0.5% near the ionisation threshold).
    Tolerances: 2e-4 where the same formula is used (the materials differ in
    the atomic mass, 207.2 vs 207.217 and 39.95 vs 39.948), 5e-3 for brems
    (Geant4's integration and gamma cut differ slightly)."""
    import geantexascalepilot_b200 as gx
    cases = [("LambdaPrim.compt.gamma", 1.0, 1e5, 2e-4), ("Lambda.compt.gamma", 0.02, 1.0, 2e-3),
             ("Lambda.eIoni.e-", 3.0, 1e5, 2e-4), ("Lambda.eIoni.e+", 3.0, 1e5, 2e-4),
             ("Lambda.eBrem.e-", 1.0, 1e3, 5e-3), ("Lambda.eBrem.e+", 1.0, 1e3, 5e-3)]
    for name, lo, hi, tol in cases:
        x, y = _nodes(name, mat)
        sel = (x >= lo) & (x <= hi) & (y > 0)
        built = dm.table_build(gx.TABLES.index(name), mat, x[sel]).cpu().numpy()
        np.testing.assert_allclose(built, y[sel], rtol=tol, err_msg=name)


@pytest.mark.parametrize("mat", [1, 2])
def test_built_pair_and_photoelectric_tables_within_their_model_bands(dm, mat):
    """Tables the reference has no per-atom cross section for, built from the
    samplers' own physics: pairs from the Bethe-Heitler differential cross
    section with Tsai's screening and triplet terms -- within 6% of the shipped
    Geant4 table from 50 MeV to 10 TeV, within 20% from 10 to 50 MeV (the Born
    approximation); photo-electric from the Sandia parameterisation -- within
    6% (lead) and 20% (argon, whose shipped table comes from another
    photo-electric model) from 200 keV up."""
    import geantexascalepilot_b200 as gx
    x, y = _nodes("Lambda.conv.gamma", mat)
    for lo, hi, tol in ((50.0, 1e7, 0.06), (10.0, 50.0, 0.2)):
        sel = (x >= lo) & (x <= hi) & (y > 0)
        built = dm.table_build(gx.TABLES.index("Lambda.conv.gamma"), mat, x[sel]).cpu().numpy()
        np.testing.assert_allclose(built, y[sel], rtol=tol)
    x, y = _nodes("LambdaPrim.phot.gamma", mat)
    sel = (x >= 0.2) & (y > 0)
    built = dm.table_build(gx.TABLES.index("LambdaPrim.phot.gamma"), mat, x[sel]).cpu().numpy()
    ratio = built / y[sel]
    if mat == 1:
        assert np.all(np.abs(ratio - 1) < 0.06)
    else:
        assert np.all((ratio > 0.8) & (ratio < 0.9))


def test_pair_integral_against_cpu(dm):
    """The device's Bethe-Heitler quadrature against the same integral in
    numpy (the sampler's screening functions, 8 x 8 Gauss-Legendre points)."""
    import geantexascalepilot_b200 as gx
    E = _grid(3.0, 1e6, 16)
    built = dm.table_build(gx.TABLES.index("Lambda.conv.gamma"), 1, E).cpu().numpy()
    Z, alpha, re = 82.0, 7.2973525376e-3, 2.8179402894e-12
    n_atoms = 6.02214179e23 * 11.35 / 207.2 * 1e-3
    az2 = (Z / 137.0) ** 2
    fc = (0.0083 * az2 * az2 + 0.20206 + 1 / (1 + az2)) * az2 - (0.0020 * az2 * az2 + 0.0369) * az2 * az2
    s1 = lambda d: np.where(d > 1, 42.24 - 8.368 * np.log(d + 0.952), 42.392 - d * (7.796 - 1.961 * d))
    s2 = lambda d: np.where(d > 1, 42.24 - 8.368 * np.log(d + 0.952), 41.405 - d * (5.828 - 0.8945 * d))
    xg, wg = np.polynomial.legendre.leggauss(8)
    xg, wg = 0.5 * (xg + 1), 0.5 * wg
    Z3 = Z ** (1 / 3)
    xi = np.log(1440 / Z3 ** 2) / (np.log(183 / Z3) - fc)
    for k, e in enumerate(E):
        eps0 = ME / e
        FZ = 8 * np.log(Z) / 3 + (8 * fc if e > 50 else 0)
        h = (0.5 - eps0) / 8
        eps = eps0 + (np.arange(8)[:, None] + xg[None, :]) * h
        u = eps * (1 - eps)
        d = 136 * eps0 / (Z3 * u)
        f = (eps ** 2 + (1 - eps) ** 2) * np.maximum(s1(d) - FZ, 0) + 2 / 3 * u * np.maximum(s2(d) - FZ, 0)
        ref = n_atoms * alpha * re * re * Z * (Z + xi) * (f * wg[None, :]).sum() * h
        assert built[k] == pytest.approx(ref, rel=1e-6)


def test_bhabha_and_brems_integrals_against_cpu(dm, oracle):
    """The device quadratures against the same integrals done in numpy
    (Bhabha analytically, Seltzer-Berger with 8 x 16 Gauss-Legendre points
    over the oracle's Seltzer-Berger table)."""
    import geantexascalepilot_b200 as gx
    pb = oracle.material(82.0, 207.2, 11.35)
    E = _grid(2.0, 500.0, 12)
    # the reference's accessor reads the file-order table at 4 ipart + index
    # (stride-4 quirk): e- in lead is entry 4, gamma in lead entry 1
    cut_e = oracle.cut_value(0, 1) * 1e-3
    cut_g = oracle.cut_value(1, 0) * 1e-3
    assert cut_e == pytest.approx(1.003864) and cut_g == pytest.approx(0.09458614)
    re = 2.8179402894e-12
    built_ep = dm.table_build(gx.TABLES.index("Lambda.eIoni.e+"), 1, E).cpu().numpy()
    built_br = dm.table_build(gx.TABLES.index("Lambda.eBrem.e-"), 1, E).cpu().numpy()
    built_bp = dm.table_build(gx.TABLES.index("Lambda.eBrem.e+"), 1, E).cpu().numpy()
    alpha = 1.0 / 137.035999679
    xg, wg = np.polynomial.legendre.leggauss(8)
    xg, wg = 0.5 * (xg + 1), 0.5 * wg
    for k, T in enumerate(E):
        gam = (T + ME) / ME
        beta2 = 1 - 1 / gam ** 2
        y = 1 / (1 + gam)
        y12 = 1 - 2 * y
        b1, b2, b4 = 2 - y * y, y12 * (3 + y * y), y12 ** 3
        b3 = b4 + y12 ** 2
        x0 = cut_e / T
        integral = (1 / x0 - 1) / beta2 - b1 * np.log(1 / x0) + b2 * (1 - x0) - b3 * (1 - x0 ** 2) / 2 + b4 * (
            1 - x0 ** 3) / 3
        assert built_ep[k] == pytest.approx(pb["n_el"] * 2 * np.pi * ME * re * re / T * integral, rel=1e-6)
        Et = T + ME
        kp2 = pb["density_factor"] * Et * Et
        v0, dv = np.log(cut_g), (np.log(T) - np.log(cut_g)) / 16
        ks = np.array([np.exp(v0 + (l + x) * dv) for l in range(16) for x in xg])
        ws = np.tile(wg, 16)
        terms = np.array([oracle.sb_value("pb", kk / T, np.log(T)) for kk in ks]) * ws / (1 + kp2 / ks ** 2)
        norm = pb["n_atoms"] * 82.0 ** 2 / (T * (T + 2 * ME) / Et ** 2) * dv * 1e-25
        assert built_br[k] == pytest.approx(norm * terms.sum(), rel=1e-9)
        # positrons: the Coulomb factor exp(2 pi alpha Z (1/beta1 - 1/beta2))
        t2 = T - ks
        ib1, ib2 = Et / np.sqrt(T * (T + 2 * ME)), (t2 + ME) / np.sqrt(t2 * (t2 + 2 * ME))
        fac = np.exp(2 * np.pi * alpha * 82.0 * (ib1 - ib2))
        assert built_bp[k] == pytest.approx(norm * (terms * fac).sum(), rel=1e-9)
        assert built_bp[k] < built_br[k]


def test_rebuilt_tables_and_computed_cuts_run_showers():
    import geantexascalepilot_b200 as gx
    from geantexascalepilot_b200 import configs
    cfg, prims, nvol = configs.c2(24)
    runs = []
    for rebuild in (False, True):
        dm = gx.ProxyDataManager()
        if rebuild:
            change = dm.rebuild_tables()
            assert change < 0.25  # the worst table: argon photo-electric (Sandia against the Geant4 build)
            dm.compute_cuts(0.7)
            v = ctypes.c_double()  # file-order entry 4 = e- in lead (see above)
            assert gx._lib.lib.gx_cut_value(dm.handle, 0, 1, ctypes.byref(v)) == 0
            assert v.value == pytest.approx(1003.8644857807957, rel=1e-12)
        cfg.precision, cfg.engine = 0, 1
        edep, st, _ = gx.transport(dm, cfg, *prims[:4], nvol=nvol)
        torch.cuda.synchronize()
        e0 = prims[1].sum()
        assert st["errors"] == 0 and abs(edep.sum().item() + st["escaped"] - e0) <= 1e-9 * e0
        runs.append((edep.cpu().numpy().reshape(-1, 2).sum(1), st))
        dm.close()
    a, b = runs[0][0], runs[1][0]
    big = a > 0.002 * a.sum()
    assert np.all(np.abs(a - b)[big] <= 5 * 0.25 / np.sqrt(24) * a[big] + 1e-3 * a.sum())
    assert abs(runs[0][1]["steps"] - runs[1][1]["steps"]) <= 0.02 * runs[0][1]["steps"]


@pytest.mark.parametrize("mat", [1, 2])
def test_built_stopping_powers_match_shipped(dm, mat):
    """Collision stopping power (Berger-Seltzer with the Sternheimer-Peierls
    density effect) within 1e-3 (argon) and 2.5% (lead, whose tabulated
    density-effect parameters differ from the general rules) above 10 keV;
    radiative loss below the gamma cut (Seltzer-Berger) within 0.3% up to
    1 GeV, for positrons (with the Coulomb factor) 1.5% below 100 keV."""
    import geantexascalepilot_b200 as gx
    tol = 2.5e-2 if mat == 1 else 1e-3
    for name in ("DEDX.eIoni.e-", "DEDX.eIoni.e+"):
        x, y = _nodes(name, mat)
        sel = (x >= 0.01) & (y > 0)
        built = dm.table_build(gx.TABLES.index(name), mat, x[sel]).cpu().numpy()
        np.testing.assert_allclose(built, y[sel], rtol=tol, err_msg=name)
    for name in ("DEDX.eBrem.e-", "DEDX.eBrem.e+"):
        x, y = _nodes(name, mat)
        sel = (x >= 0.01) & (x <= 1e3) & (y > 0)
        built = dm.table_build(gx.TABLES.index(name), mat, x[sel]).cpu().numpy()
        # positrons below 100 keV, where the Coulomb factor cuts the loss to
        # 8-80% of the electrons': the factor's ratio to Geant4's is within 1%
        tol = np.where((x[sel] < 0.1) & (name[-1] == "+"), 1.5e-2, 3e-3)
        assert np.all(np.abs(built / y[sel] - 1) <= tol), (name, np.max(np.abs(built / y[sel] - 1)))


def test_rebuilt_ranges_and_inverse_ranges():
    """After gx_ctx_rebuild_tables the range tables integrate the rebuilt
    losses: within 2e-3 of the shipped argon ranges and 4% of the lead ones,
    and the inverse range maps each range back to its energy."""
    import geantexascalepilot_b200 as gx
    dm = gx.ProxyDataManager()
    dm.rebuild_tables()
    for mat, tol in ((1, 0.04), (2, 2e-3)):
        for ep, rname, iname in ((0, "Range.eIoni.e-", "InverseRange.eIoni.e-"),
                                 (1, "Range.eIoni.e+", "InverseRange.eIoni.e+")):
            x, y = _nodes(rname, mat)
            r = dm.table_value(gx.TABLES.index(rname), mat, x).cpu().numpy()
            np.testing.assert_allclose(r, y, rtol=tol, err_msg=rname)
            e = dm.inv_range_value(gx.TABLES.index(iname), mat, r).cpu().numpy()
            np.testing.assert_allclose(e, x, rtol=1e-9, err_msg=iname)
    dm.close()
