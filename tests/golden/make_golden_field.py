#!/usr/bin/env python3
"""Golden vectors for the field map, from the reference's own reader
(examples/magneticfield/simplifiedCMS/inc/Geant/ScalarCMSmagField.h, compiled
in place through oracle/refshim_field into oracle/_ref/libgxref_field.so by
oracle/build_ref.sh), reading the shipped map
(geantexascalepilot_b200/data/field/cmsmagfield2015.txt).

field.npz: 2000 seeded points (inside the lattice, beyond it in r and z, on
the axis, on lattice lines) and the field there, tesla.

Usage: python tests/golden/make_golden_field.py
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SO = os.path.join(ROOT, "oracle", "_ref", "libgxref_field.so")
MAP = os.path.join(ROOT, "geantexascalepilot_b200", "data", "field", "cmsmagfield2015.txt")


def points(rng):
    n = 1600
    r = rng.uniform(0, 9000, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    z = rng.uniform(-16000, 16000, n)
    p = [np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)]
    p.append(np.stack([np.zeros(50), np.zeros(50), rng.uniform(-16000, 16000, 50)], 1))        # axis
    p.append(np.stack([rng.uniform(9000, 12000, 50), np.zeros(50), rng.uniform(-2e4, 2e4, 50)], 1))  # outside
    g = np.stack([50.0 * rng.integers(0, 181, 150), np.zeros(150), -16000 + 200.0 * rng.integers(0, 161, 150)], 1)
    p.append(g)                                                                                  # lattice points
    p.append(np.stack([rng.uniform(-400, 400, 150), rng.uniform(-400, 400, 150), rng.uniform(-400, 400, 150)], 1))
    return np.concatenate(p)


def main():
    lib = C.CDLL(SO)
    lib.gxref_field_load.argtypes = [C.c_char_p]
    lib.gxref_field_value.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.gxref_field_load(MAP.encode())
    pos = np.ascontiguousarray(points(np.random.default_rng(20241204)))
    B = np.zeros_like(pos)
    lib.gxref_field_value(len(pos), pos.ctypes.data_as(C.POINTER(C.c_double)), B.ctypes.data_as(C.POINTER(C.c_double)))
    np.savez_compressed(os.path.join(HERE, "field.npz"), pos=pos, B=B)
    print("field.npz:", pos.shape, "B at origin", B[np.argmin(np.linalg.norm(pos, axis=1))])


if __name__ == "__main__":
    main()
