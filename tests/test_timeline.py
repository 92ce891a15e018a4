"""The timeline tracing interface: the product library refuses it (its kernels
carry no tracing code), and the summary of a record (CPU only)."""
import numpy as np


def test_product_library_has_no_timeline():
    from geantexascalepilot_b200._lib import GX_ERR_ARG, lib
    assert lib.gx_timeline_reset(None) == GX_ERR_ARG
    assert b"GX_TIMELINE" in lib.gx_last_error_string()
    assert lib.gx_timeline_read(None, None, 0) == GX_ERR_ARG


def test_summary_of_a_record():
    from geantexascalepilot_b200 import timeline as T
    a = np.full((T.ROWS, T.KERNELS, 2), np.uint64(0), dtype=np.uint64)
    a[:, :, 0] = np.uint64(0xFFFFFFFFFFFFFFFF)

    def put(row, k, s_us, e_us, base):
        a[row, k, 0] = np.uint64(base + s_us * 1000)
        a[row, k, 1] = np.uint64(base + e_us * 1000)

    # the planning launch (row 0) is not an iteration
    put(0, 14, 0, 1, 0)
    # iteration 0: the e+ chain ends last; iteration 1 (3 ms): the gamma chain
    base = 10 ** 9
    for k, s, e in ((0, 0, 2), (1, 2, 3), (2, 3, 50), (3, 3, 40), (4, 3, 60), (5, 50, 55), (8, 40, 45),
                    (11, 60, 70), (14, 70, 72)):
        put(1, k, s, e, base)
    base2 = base + 100_000
    for k, s, e in ((0, 0, 2), (1, 2, 3), (2, 3, 2900), (3, 3, 100), (4, 3, 50), (5, 2900, 2990),
                    (14, 2990, 3000)):
        put(2, k, s, e, base2)
    r = T.summary(a, iterations=2)
    assert r["iterations"] == 2
    assert r["chain_ending_the_iteration"] == {"gamma": 1, "e-": 0, "e+": 1}
    assert abs(r["sum_of_iteration_spans_ms"] - 3.072) < 1e-9
    assert abs(r["wall_ms"] - 3.1) < 1e-9
    assert r["iterations_over_2ms"] == 1
    assert r["kernels"]["transport gamma"]["launches"] == 2
    assert abs(r["kernels"]["transport gamma"]["max_us"] - 2897.0) < 1e-9
    assert r["some_kernel_running_frac"] == 1.0
    assert r["longest_iteration"]["iteration"] == 1
    try:
        T.summary(a, iterations=T.ROWS)
    except ValueError:
        pass
    else:
        raise AssertionError("a run longer than the record must be refused")
