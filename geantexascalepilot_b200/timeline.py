"""Timeline tracing of the batched engine (the library's tracing build).

With lib/libgxb200_timeline.so loaded (build it with
``python geantexascalepilot_b200/build.py --timeline`` and point GX_LIB_PATH
at it), every step kernel of the batched engine records the GPU global timer
at the start of its first block and at the end of its last, per iteration:
``reset`` clears the record, ``read`` returns it as an array
[512 iterations, 16 kernels, (start, end)] in nanoseconds, and ``summary``
condenses it: how long the iterations take, how much of the time some kernel
runs, how long each kernel runs, and which particle type's chain (its
transport kernel and then its interaction kernels) ends each iteration.
The reference traces with timemory markers (TIMEMORY_* in its sources); this
is the same kind of record for the GPU kernels, kept out of the product
library so that the product's kernels carry no tracing code.
"""
import ctypes as C

import numpy as np

from ._lib import check, lib

ROWS, KERNELS = 512, 16
NAMES = ["refill", "refill bookkeeping", "transport gamma", "transport e-", "transport e+",
         "Compton", "conversion", "photo-electric", "Moller", "e- bremsstrahlung", "(unused)",
         "Bhabha", "e+ bremsstrahlung", "annihilation", "end of iteration", "(unused)"]
CHAINS = {"gamma": (2, 5, 6, 7), "e-": (3, 8, 9), "e+": (4, 11, 12, 13)}
_UNSET = np.uint64(0xFFFFFFFFFFFFFFFF)


def reset(dm):
    """Clear the record (gx_timeline_reset); raises GxError with the product library."""
    check(lib.gx_timeline_reset(dm.handle))


def read(dm):
    """The record after a device synchronisation: uint64 [ROWS, KERNELS, 2]."""
    buf = (C.c_ulonglong * (ROWS * KERNELS * 2))()
    check(lib.gx_timeline_read(dm.handle, C.cast(buf, C.c_void_p), ROWS * KERNELS * 2))
    return np.frombuffer(buf, dtype=np.uint64).reshape(ROWS, KERNELS, 2).copy()


def _union(iv):
    iv = sorted(iv)
    tot, (cs, ce) = 0.0, iv[0]
    for s, e in iv[1:]:
        if s > ce:
            tot += ce - cs
            cs, ce = s, e
        else:
            ce = max(ce, e)
    return tot + ce - cs


def summary(a, iterations=None):
    """Condensed record of one run: a = read(dm) after a run of `iterations`
    iterations (at most ROWS - 1: the rows are reused modulo ROWS)."""
    if iterations is not None and iterations > ROWS - 1:
        raise ValueError("the record keeps %d iterations; this run took %d" % (ROWS - 1, iterations))
    ran = a[:, :, 0] != _UNSET
    rows = [r for r in range(1, ROWS) if ran[r, 0] and ran[r, 14]]
    if not rows:
        return {"iterations": 0}
    t = a.astype(np.float64)
    spans, busy = [], 0.0
    per = {k: [] for k in range(KERNELS)}
    crit = {c: 0 for c in CHAINS}
    for r in rows:
        ks = [k for k in range(KERNELS) if ran[r, k]]
        spans.append(t[r, 14, 1] - t[r, 0, 0])
        busy += _union([(t[r, k, 0], t[r, k, 1]) for k in ks])
        for k in ks:
            per[k].append(t[r, k, 1] - t[r, k, 0])
        ends = {c: max((t[r, k, 1] for k in ks_ if ran[r, k]), default=0.0) for c, ks_ in CHAINS.items()}
        crit[max(ends, key=ends.get)] += 1
    spans = np.array(spans)
    wall = t[rows[-1], 14, 1] - t[rows[0], 0, 0]
    big = spans > 2e6
    r_max = rows[int(np.argmax(spans))]
    t0 = t[r_max, 0, 0]
    return {
        "iterations": len(rows),
        "wall_ms": wall / 1e6,
        "sum_of_iteration_spans_ms": float(spans.sum()) / 1e6,
        "some_kernel_running_frac": busy / float(spans.sum()),
        "iterations_over_2ms": int(big.sum()),
        "time_share_of_iterations_over_2ms": float(spans[big].sum() / spans.sum()),
        "kernels": {NAMES[k]: {"launches": len(v), "total_ms": float(np.sum(v)) / 1e6,
                               "mean_us": float(np.mean(v)) / 1e3, "max_us": float(np.max(v)) / 1e3}
                    for k, v in per.items() if v},
        "chain_ending_the_iteration": crit,
        "longest_iteration": {"iteration": r_max - 1, "span_us": float(spans.max()) / 1e3,
                              "kernels_us": {NAMES[k]: [round((t[r_max, k, 0] - t0) / 1e3, 1),
                                                        round((t[r_max, k, 1] - t0) / 1e3, 1)]
                                             for k in range(KERNELS) if ran[r_max, k]}},
    }
