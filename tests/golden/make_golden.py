#!/usr/bin/env python3
"""Generate the golden vectors in this directory from the reference's own code.

Runs the reference's hot-path sources compiled in place
(oracle/_ref/libgxref.so, built by oracle/build_ref.sh from a reference
checkout) on seeded inputs and stores inputs and outputs as .npz fixtures.
The reference has no golden vectors or known-answer tests of its own for this
path, so these outputs are the pin for the oracle and the CUDA kernels.

Usage: python tests/golden/make_golden.py   (needs the reference checkout)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_ctypes import Oracle, Reference  # noqa: E402

SEED = np.full(6, 12345.0)
DATA = os.path.join(os.path.dirname(os.path.dirname(HERE)), "geantexascalepilot_b200", "data")


def _vectors(fn):
    """bin (x) vectors of a Geant4-format ASCII physics table"""
    t = open(fn).read().split()
    i, out = 1, []
    for _ in range(int(t[0])):
        siz = int(t[i + 4])
        i += 5
        out.append(np.array(t[i:i + 2 * siz], dtype=float).reshape(siz, 2)[:, 0])
        i += 2 * siz
    return out


def unit_dirs(rng, n):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    # axis-aligned edge cases for RotateToLabFrame (up == 0, u3 < 0)
    v[:4] = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [0, 1, 0]]
    return v


def main():
    ref = Reference()
    orc = Oracle()  # only to derive substream states; its outputs are not stored
    rng = np.random.default_rng(20240603)

    # ---------------------------------------------------------------- MRG32k3a
    draws, state = ref.mrg_draws(SEED, 1000)
    sid = np.stack([ref.stream_id_draws(i, 4) for i in range(0, 4)])
    adv_cases = np.array([[76, 0], [127, 0], [0, 1], [0, 12345], [5, -3], [-4, 9], [40, 7], [0, -1]])
    adv = np.stack([ref.advance(SEED, int(e), int(c)) for e, c in adv_cases])
    sub = {}
    for s in (12345.0, 2024.0, 7.0):
        st = np.full(6, s)
        states = [st.copy()]
        for _ in range(7):
            states.append(ref.advance(states[-1], 76, 0))
        sub[str(int(s))] = np.stack(states)
    np.savez_compressed(os.path.join(HERE, "mrg.npz"), seed=SEED, draws=draws, state_after=state,
                        stream_id_draws=sid, adv_cases=adv_cases, adv=adv,
                        substreams_12345=sub["12345"], substreams_2024=sub["2024"], substreams_7=sub["7"])

    # ------------------------------------------------------------------ tables
    ref.init_tables()
    E = np.concatenate([np.logspace(-4.5, 8.5, 400), [1e-4, 1.0, 0.2, 1.02199782, 1e8]])
    tab_vals = np.zeros((20, 3, E.size))
    for t in range(20):
        for m in range(3):
            tab_vals[t, m] = ref.table_value(t, m, E)
    R = np.logspace(-7, 10, 400)
    inv_vals = np.zeros((2, 3, R.size))
    for k, t in enumerate((4, 5)):
        for m in range(3):
            inv_vals[k, m] = ref.table_invrange(t, m, R)
    cuts = np.array([[ref.cut_value(i, p) for p in range(3)] for i in range(3)])
    sbx = rng.uniform(-0.1, 1.1, 300)
    sby = rng.uniform(-8.0, 10.0, 300)
    sbv = np.array([[ref.sb2d_value(z, x, y) for x, y in zip(sbx, sby)] for z in (11, 18, 82)])
    # Value() on the range-indexed InverseRange vectors is undefined in the
    # reference (its bin search leaves the vector), so those rows are not pinned.
    np.savez_compressed(os.path.join(HERE, "tables.npz"), E=E, values=tab_vals, R=R, invrange=inv_vals,
                        cuts=cuts, sb_x=sbx, sb_y=sby, sb_values=sbv, sb_Z=np.array([11, 18, 82]))

    # ------------------------------------------------------------------ models
    n = 256
    ranges = {"kn": (1e-4, 1e5), "sg": (1e-4, 1e2), "bh": (1.03, 1e5), "sb": (2e-3, 1e5), "mb": (3e-3, 1e5)}
    out = {}
    for k, (model, (lo, hi)) in enumerate(ranges.items()):
        states = orc.substreams(SEED, 100 * k, n)
        Ein = 10 ** rng.uniform(np.log10(lo), np.log10(hi), n)
        D = unit_dirs(rng, n)
        r = ref.interact(model, states, Ein, D)
        out[model + "_states"] = states
        out[model + "_E_in"] = Ein
        out[model + "_dir_in"] = D
        for key in ("E", "dir", "edep", "status", "nsec", "sec_type", "sec_E", "sec_dir"):
            out[model + "_" + key] = r[key]
        out[model + "_states_out"] = r["states"]
    np.savez_compressed(os.path.join(HERE, "models_quirk.npz"), **out)

    # ------------------------------------------------- cross sections / helpers
    Zs = np.array([1.0, 10.0, 18.0, 82.0])
    Exs = np.logspace(-5.5, 5, 60)
    kn = np.array([[ref.lib.gxref_kn_xs(z, e) for e in Exs] for z in Zs])
    mb = np.array([[ref.lib.gxref_mb_xs(z, e) for e in Exs] for z in Zs])
    Esg = np.logspace(-5, 0, 80)
    sg = np.array([[ref.lib.gxref_sg_photo_energy(z, e) for e in Esg] for z in (10, 18, 82)])
    coul = np.array([ref.lib.gxref_coulomb(z) for z in Zs])
    np.savez_compressed(os.path.join(HERE, "xs.npz"), Z=Zs, E=Exs, kn=kn, mb=mb, E_sg=Esg, sg=sg, coulomb=coul)

    # --------------------------------------------------------------- processes
    m = 500
    gp_states = orc.substreams(SEED, 7000, m)
    proc = np.arange(m) % 5
    gp_E = 10 ** rng.uniform(-3, 5, m)
    gp_nil = np.where(np.arange(m) % 3 == 0, -1.0, np.where(np.arange(m) % 3 == 1, 0.0, rng.uniform(0.1, 3, m)))
    gp_saved = rng.uniform(0.1, 100, m)
    gp_ps = rng.uniform(0, 10, m)
    res = [ref.post_step_gpil(int(p), s, e, ps, nl, sv, mat=2)
           for p, s, e, ps, nl, sv in zip(proc, gp_states, gp_E, gp_ps, gp_nil, gp_saved)]
    ag_mat = np.arange(600) % 3
    ag_E = 10 ** rng.uniform(-4.5, 5, 600)
    ag = np.array([ref.ioni_along_gpil(int(mt), e) for mt, e in zip(ag_mat, ag_E)])
    ad_mat = 1 + np.arange(600) % 2
    ad_E = 10 ** rng.uniform(-4.5, 4, 600)
    rg = np.array([orc.table_value(18, int(mt), np.array([e]))[0] for mt, e in zip(ad_mat, ad_E)])
    ad_step = rg * rng.choice([0.001, 0.005, 0.05, 0.3, 0.9, 1.2], 600)
    ad = np.array([ref.ioni_along_doit(int(mt), s, e) for mt, s, e in zip(ad_mat, ad_step, ad_E)])
    # Where the loss exceeds 1% the reference reads the inverse range through
    # Value(), whose log-grid bin can leave the range-indexed vector; mark the
    # cases whose lookup stays inside it (the only ones with a defined result).
    inv_x = _vectors(os.path.join(DATA, "table", "InverseRange.eIoni.e-.asc"))
    dedx = np.array([orc.table_value(2, int(mt), np.array([e]))[0] for mt, e in zip(ad_mat, ad_E)])
    defined = np.ones(600, dtype=bool)
    for i in range(600):
        if ad_step[i] < rg[i] and ad_E[i] > 1e-4 and ad_step[i] * dedx[i] > 0.01 * ad_E[i]:
            x = inv_x[int(ad_mat[i])]
            r_left = rg[i] - ad_step[i]
            if x[0] < r_left < x[-1]:
                dbin = np.log(x[1] / x[0])
                defined[i] = int(np.log(r_left) / dbin - np.log(x[0]) / dbin) <= x.size - 2
    np.savez_compressed(os.path.join(HERE, "processes.npz"), gpil_proc=proc, gpil_states=gp_states, gpil_E=gp_E,
                        gpil_nil=gp_nil, gpil_saved=gp_saved, gpil_pstep=gp_ps,
                        gpil_step=np.array([x[0] for x in res]), gpil_nil_out=np.array([x[1] for x in res]),
                        gpil_saved_out=np.array([x[2] for x in res]), gpil_states_out=np.stack([x[3] for x in res]),
                        agpil_mat=ag_mat, agpil_E=ag_E, agpil_step=ag, adoit_mat=ad_mat, adoit_E=ad_E,
                        adoit_step=ad_step, adoit_E_out=ad[:, 0], adoit_edep=ad[:, 1],
                        adoit_defined=defined)

    # ------------------------------------------------------------------- helix
    h = 500
    B = np.array([0.3, -0.2, 30.0])
    pos = rng.normal(size=(h, 3)) * 10
    D = unit_dirs(rng, h)
    ch = rng.choice([-1.0, 1.0], h)
    mom = 10 ** rng.uniform(-3, 2, h)
    st = 10 ** rng.uniform(-4, 2, h)
    npos, ndir = ref.helix(B, pos, D, ch, mom, st)
    np.savez_compressed(os.path.join(HERE, "helix.npz"), B=B, pos=pos, dir=D, charge=ch, mom=mom, step=st,
                        newpos=npos, newdir=ndir)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
