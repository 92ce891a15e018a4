"""Build the CUDA library of this package in-tree.

Compiles every csrc/*.cu for sm_100a (B200) with nvcc and links
geantexascalepilot_b200/lib/libgxb200.so.  Nothing is JIT-compiled at run
time; the library is loaded with ctypes by geantexascalepilot_b200._lib.

    python geantexascalepilot_b200/build.py [-v] [--timeline]

--timeline builds the tracing variant instead, lib/libgxb200_timeline.so
(objects in _build_timeline/): the same sources with GX_TIMELINE defined for
the transport engine, whose step kernels then record when each kernel of an
iteration starts and ends (gx_timeline_read).  Load it in place of the
product with GX_LIB_PATH, e.g. for `python -m geantexascalepilot_b200.run c3
--timeline out.npy`.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
BUILD = os.path.join(os.path.dirname(PKG), "_build")
LIB = os.path.join(LIBDIR, "libgxb200.so")
BUILD_TIMELINE = os.path.join(os.path.dirname(PKG), "_build_timeline")
LIB_TIMELINE = os.path.join(LIBDIR, "libgxb200_timeline.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wno-unused-function"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def system_libstdcxx():
    """The shared libstdc++ the host process uses: a static copy inside a
    library that is loaded next to another libstdc++ breaks iostream set-up."""
    for c in ("/usr/lib/x86_64-linux-gnu/libstdc++.so.6", "/lib/x86_64-linux-gnu/libstdc++.so.6"):
        if os.path.exists(c):
            return c
    return None


# The per-function batch kernels, the particle gun and the FP64 parity variant
# of the transport reproduce FP64 host arithmetic operation by operation: no
# fused multiply-adds there, so they round like the host code.  The transport
# engine itself keeps contraction.
PER_FILE = {"gx_kernels.cu": ["-fmad=false"], "gx_events.cu": ["-fmad=false"],
            "gx_transport_parity.cu": ["-fmad=false"]}


def _includes(src, seen=None):
    """src and the files of csrc/ it includes, directly or through others."""
    seen = set() if seen is None else seen
    if src in seen or not os.path.exists(src):
        return seen
    seen.add(src)
    with open(src) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include \""):
                _includes(os.path.join(CSRC, line.split('"')[1]), seen)
    return seen


def _compile(src, verbose, build_dir=BUILD, timeline=False):
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    # the source, every header of the directory (headers include one another),
    # the .cu files it includes, the ABI header and this script
    deps = (sorted(_includes(src)) + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
            [os.path.join(os.path.dirname(PKG), "include", "gx_abi.h"), os.path.abspath(__file__)])
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    extra = PER_FILE.get(os.path.basename(src), [])
    if timeline and os.path.basename(src) == "gx_transport.cu":
        extra = extra + ["-DGX_TIMELINE"]
    cmd = [nvcc()] + ARCH + FLAGS + extra + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(verbose=False, timeline=False):
    build_dir, lib = (BUILD_TIMELINE, LIB_TIMELINE) if timeline else (BUILD, LIB)
    os.makedirs(build_dir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, build_dir, timeline), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if os.path.exists(lib) and os.path.getmtime(lib) >= max(os.path.getmtime(o) for o in objs):
        return lib
    cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    cxx = system_libstdcxx()
    if cxx:
        cmd += ["-Xlinker", cxx]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, timeline="--timeline" in sys.argv))
