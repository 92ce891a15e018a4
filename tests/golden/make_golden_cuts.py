#!/usr/bin/env python3
"""Golden vectors for the production-cut converter, from the reference's own
code (source/Geant/cuts compiled in place through oracle/refshim_cuts into
oracle/_ref/libgxref_cuts.so by oracle/build_ref.sh).

cuts.npz: for the materials of the calorimeter (vacuum, lead, liquid argon)
and a two-element compound, every particle (gamma, e-, e+) and a range of
cuts: the energy of a length cut and the length of an energy cut.

Usage: python tests/golden/make_golden_cuts.py
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "libgxref_cuts.so")
AVOGADRO = 6.02214179e+23

# name, Z, A (g/mol), atoms per formula unit, density (g/cm3)
MATERIALS = [("Galactic", [1.0], [1.01], [1], 1e-25), ("Pb", [82.0], [207.2], [1], 11.35),
             ("LAr", [18.0], [39.95], [1], 1.396), ("CO2-like", [6.0, 8.0], [12.011, 15.999], [1, 2], 1.8)]
CUTS_MM = [0.001, 0.01, 0.1, 0.7, 1.0, 10.0, 1000.0]
CUTS_MEV = [1e-4, 1e-3, 0.01, 0.1, 1.0, 100.0, 2e4]


def atoms_per_mm3(A, nat, rho):
    mol = sum(a * k for a, k in zip(A, nat))  # g per mole of formula units
    return [AVOGADRO * rho / mol * k * 1e-3 for k in nat]


def main():
    lib = C.CDLL(SO)
    D = C.c_double
    lib.gxref_cut_elements.argtypes = [C.c_int, C.POINTER(D)]
    lib.gxref_cut_convert.restype = D
    lib.gxref_cut_convert.argtypes = [C.c_int, C.c_int, C.POINTER(D), C.POINTER(D), D, D, C.c_int]
    allZ = sorted({z for _, Z, _, _, _ in MATERIALS for z in Z})
    lib.gxref_cut_elements(len(allZ), (D * len(allZ))(*allZ))
    out = {"cuts_mm": np.array(CUTS_MM), "cuts_mev": np.array(CUTS_MEV), "names": np.array([m[0] for m in MATERIALS])}
    for name, Z, A, nat, rho in MATERIALS:
        n = atoms_per_mm3(A, nat, rho)
        z, na = (D * len(Z))(*Z), (D * len(n))(*n)
        out[name + "_Z"], out[name + "_n"], out[name + "_rho"] = np.array(Z), np.array(n), rho
        out[name + "_energy"] = np.array([[lib.gxref_cut_convert(p, len(Z), z, na, rho, c, 1) for c in CUTS_MM]
                                          for p in range(3)])
        out[name + "_length"] = np.array([[lib.gxref_cut_convert(p, len(Z), z, na, rho, c, 0) for c in CUTS_MEV]
                                          for p in range(3)])
    np.savez_compressed(os.path.join(HERE, "cuts.npz"), **out)
    print("cuts.npz:", sorted(out))


if __name__ == "__main__":
    main()
