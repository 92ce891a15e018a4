#!/usr/bin/env python3
"""Import the physics data that the reference ships with its EM transport path.

The reference reads its Geant4-format ASCII physics tables, cut table,
Seltzer-Berger bremsstrahlung tables and (in its field example) the CMS
field map at run time from
``source/Geant/proxy/test/BasicCpuTransport/data/`` (see
``source/Geant/proxy/src/ProxyDataManager.cu:49-122`` and
``source/Geant/proxy/ProxySeltzerBerger.hpp:134-152``).  This script copies
the subset this framework loads into the package's data directory
(``geantexascalepilot_b200/data``), unchanged, and extracts
the atomic-shell and Sandia photo-absorption arrays that the reference keeps
as C++ data tables in ``source/Geant/proxy/ProxySandiaData.hpp`` into a plain
text file (``sandia.dat``) so that nothing here has to include reference code.

Usage:  python import_reference_data.py <reference-checkout-root>

The files written are data, not code; they are committed so that the GPU
runs, which have no reference checkout, can load them.
"""
import os
import re
import shutil
import sys

HERE = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                    "geantexascalepilot_b200", "data")

TABLES = [
    "DEDX.eBrem.e-.asc", "DEDX.eBrem.e+.asc", "DEDX.eIoni.e-.asc", "DEDX.eIoni.e+.asc",
    "InverseRange.eIoni.e-.asc", "InverseRange.eIoni.e+.asc",
    "Ionisation.eIoni.e-.asc", "Ionisation.eIoni.e+.asc",
    "Lambda.compt.gamma.asc", "Lambda.conv.gamma.asc",
    "Lambda.eBrem.e-.asc", "Lambda.eBrem.e+.asc", "Lambda.eIoni.e-.asc", "Lambda.eIoni.e+.asc",
    "LambdaMod1.msc.e-.asc", "LambdaMod1.msc.e+.asc",
    "LambdaPrim.compt.gamma.asc", "LambdaPrim.phot.gamma.asc",
    "Range.eIoni.e-.asc", "Range.eIoni.e+.asc",
    "cut.dat", "couple.dat",
]
# Seltzer-Berger files: br<Z>.  Z=11 is the table the reference's hard-coded
# slot 10 reads (ProxySeltzerBerger.hpp:141-144,222); 18 (Ar) and 82 (Pb) are
# the calorimeter materials.
SB_Z = [11, 18, 82]


def _array_body(src, name):
    m = re.search(r"\b%s\s*\[[^\]]*\](\s*\[[^\]]*\])?\s*=\s*\{" % re.escape(name), src)
    if not m:
        raise RuntimeError("array %s not found" % name)
    i = m.end()
    depth = 1
    j = i
    while depth:
        c = src[j]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
        j += 1
    body = src[i:j - 1]
    body = re.sub(r"//[^\n]*", "", body)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return body


def _numbers(body):
    return [float(t) for t in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?", body)]


def main(ref_root):
    data = os.path.join(ref_root, "source/Geant/proxy/test/BasicCpuTransport/data")
    os.makedirs(os.path.join(HERE, "table"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "brem_SB"), exist_ok=True)
    for t in TABLES:
        shutil.copyfile(os.path.join(data, "table", t), os.path.join(HERE, "table", t))
    for z in SB_Z:
        shutil.copyfile(os.path.join(data, "brem_SB", "br%d" % z), os.path.join(HERE, "brem_SB", "br%d" % z))
    # the CMS solenoid field map of the reference's field example (181 x 161
    # (r, z) points, read by examples/magneticfield/simplifiedCMS/inc/Geant/
    # ScalarCMSmagField.h)
    os.makedirs(os.path.join(HERE, "field"), exist_ok=True)
    shutil.copyfile(os.path.join(ref_root, "examples/magneticfield/simplifiedCMS/cmsmagfield2015.txt"),
                    os.path.join(HERE, "field", "cmsmagfield2015.txt"))

    src = open(os.path.join(ref_root, "source/Geant/proxy/ProxySandiaData.hpp")).read()
    nshell = [int(v) for v in _numbers(_array_body(src, "fNumberOfShells"))]
    ishell = [int(v) for v in _numbers(_array_body(src, "fIndexOfShells"))]
    bind = _numbers(_array_body(src, "fBindingEnergies"))
    nint = [int(v) for v in _numbers(_array_body(src, "fNbOfIntervals"))]
    table = _numbers(_array_body(src, "fSandiaTable"))
    assert len(nshell) == 101 and len(ishell) == 101 and len(bind) == 1540, (len(nshell), len(ishell), len(bind))
    # rows the reference leaves out of the initialiser are zero-initialised
    assert len(nint) == 101 and len(table) % 5 == 0 and len(table) <= 981 * 5, (len(nint), len(table))
    assert sum(nint) + 1 <= len(table) // 5
    table += [0.0] * (981 * 5 - len(table))
    with open(os.path.join(HERE, "sandia.dat"), "w") as f:
        f.write("# atomic shells and Sandia photo-absorption coefficients, extracted from the\n")
        f.write("# reference's ProxySandiaData.hpp by import_reference_data.py\n")
        f.write("# units: binding energies eV; Sandia rows {edge keV, a1..a4 in cm2 keV^k / g}\n")
        f.write("SHELLS 101\n")
        f.write(" ".join(str(v) for v in nshell) + "\n")
        f.write(" ".join(str(v) for v in ishell) + "\n")
        f.write("BINDING %d\n" % len(bind))
        for k in range(0, len(bind), 8):
            f.write(" ".join(repr(v) for v in bind[k:k + 8]) + "\n")
        f.write("INTERVALS 101\n")
        f.write(" ".join(str(v) for v in nint) + "\n")
        f.write("SANDIA 981\n")
        for r in range(981):
            f.write(" ".join(repr(v) for v in table[5 * r:5 * r + 5]) + "\n")
    print("imported data into", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
