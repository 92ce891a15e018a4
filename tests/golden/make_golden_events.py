#!/usr/bin/env python3
"""Golden vectors for the event generators, from the reference's own code.

Writes
  hepevt_sample.data  a synthetic HEPEVT ASCII file (seeded decay trees of
                      made-up events: documentation entries, decayed
                      intermediates, final-state photons, electrons,
                      positrons, pions, muons, protons; an orphan final-state
                      entry; momenta and masses in GeV)
  events.npz          the reference's ProxyEgammaGun output for two gun
                      settings (from the default stream and from a
                      mid-stream state), its SetDirectionXYZ directions, and
                      its ProxyHepEvtGenerator output for the sample file

The reference code runs compiled in place (oracle/_ref/libgxref.so, built by
oracle/build_ref.sh).  Usage: python tests/golden/make_golden_events.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_ctypes import Reference  # noqa: E402

MASS = {22: 0.0, 11: 0.000510998910, -11: 0.000510998910, 13: 0.1056583745, -13: 0.1056583745, 211: 0.13957018,
        -211: 0.13957018, 111: 0.1349766, 2212: 0.938272046, 23: 91.1876, 221: 0.547862}


def _vec(rng, pmag):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v) * pmag


def make_hepevt(path, nevents, rng):
    """Seeded decay trees: entry 1 a boson (status 2) decaying to 2-5
    daughters; some daughters (pi0, eta) decay again to photons or e+e-."""
    lines = []
    for _ in range(nevents):
        ent = []  # [ist, id, jda1, jda2, px, py, pz, m]
        ent.append([2, 23, 0, 0, *(_vec(rng, rng.uniform(0, 20))), MASS[23]])
        nd = int(rng.integers(2, 6))
        first = len(ent) + 1
        for _ in range(nd):
            pid = int(rng.choice([22, 11, -11, 211, -211, 13, -13, 111, 221, 2212]))
            ent.append([1, pid, 0, 0, *(_vec(rng, rng.uniform(0.5, 50))), MASS[pid]])
        ent[0][2], ent[0][3] = first, first + nd - 1
        # second generation
        for i in range(first - 1, first - 1 + nd):
            if ent[i][1] in (111, 221):
                ent[i][0] = 2
                kids = [22, 22] if rng.random() < 0.8 else [11, -11]
                ent[i][2], ent[i][3] = len(ent) + 1, len(ent) + len(kids)
                for k in kids:
                    ent.append([1, k, 0, 0, *(_vec(rng, rng.uniform(0.1, 20))), MASS[k]])
        if rng.random() < 0.5:  # a final-state entry that is nobody's daughter
            ent.append([1, 22, 0, 0, *(_vec(rng, rng.uniform(1, 5))), 0.0])
        lines.append("%d" % len(ent))
        for e in ent:
            lines.append("%d %d %d %d %.9e %.9e %.9e %.9e" % tuple(e))
    open(path, "w").write("\n".join(lines) + "\n")


def main():
    ref = Reference()
    rng = np.random.default_rng(20241203)
    out = {}
    two_pi = 2 * np.pi
    guns = [
        # name, state, nevents, nparticles, gamma fraction, p range (MeV), eta range, phi range
        ("gun_default", np.full(6, 12345.0), 4, 25, 0.5, 1000.0, 1.0e6, -3.0, 3.0, 0.0, two_pi),
        ("gun_narrow", np.array([1., 2., 3., 4., 5., 6.]) * 98765.0, 3, 40, 0.3, 10.0, 1.0e5, 1.5, 2.5, -0.2, 0.2),
    ]
    for name, st, ne, npart, gf, p0, p1, e0, e1, f0, f1 in guns:
        pdg, p, ek, d, st_out = ref.egamma_gun(st, ne, npart, gf, p0, p1, e0, e1, f0, f1)
        out[name + "_params"] = np.array([ne, npart, gf, p0, p1, e0, e1, f0, f1])
        out[name + "_state"] = st
        out[name + "_state_out"] = st_out
        out[name + "_pdg"] = pdg
        out[name + "_p"] = p
        out[name + "_ekin"] = ek
        out[name + "_dir"] = d
    xyz = np.array([[1.0, 0.5, 2.0], [0.0, 0.0, 1.0], [0.3, -0.4, 5.0], [-1.0, 2.0, 0.5]])
    out["dir_xyz"] = xyz
    out["dir_ref"] = np.stack([ref.egamma_direction(*v) for v in xyz])
    hep = os.path.join(HERE, "hepevt_sample.data")
    make_hepevt(hep, 12, rng)
    h = ref.hepevt(hep, 12)
    for k, v in h.items():
        out["hepevt_" + k] = v
    np.savez_compressed(os.path.join(HERE, "events.npz"), **out)
    print("events.npz:", {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
