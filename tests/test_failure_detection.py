"""Failure detection on the host, by injection: the stage-two search fed
rejected evaluations (the reference's own StageTwoSearch tests,
src/sc/nebula.rs:3515-3600), BOBYQA's evaluation budget running out
(src/numeric/bobyqa.rs:778, MAXEVAL_REACHED), and non-finite inputs refused
at the C-ABI before any device work (src/sc/nebula.rs:539, 574; the design
check of nebula_sparse_with). The device side, a wait for work that runs
out, is tests/test_gpu_ring.py."""
import ctypes
import math

import numpy as np
import pytest

from edge_rs_b200 import NebulaError, _ffi, nebula_sparse_cuda

lib = _ffi.product_library()


def arr(values):
    return (ctypes.c_double * len(values))(*values)


def run_search(start, ord, f, lower=None, upper=None):
    """Drives nb_search with f(x, order, calls) as the reference's run_search
    does (nebula.rs:3515-3541); returns (found, x, failed, order)."""
    n = len(start)
    lower = lower or [1e-4] * n
    upper = upper or ([10.0, 1000.0] if n == 2 else [10.0])
    h = lib.nb_search_new(arr(start), arr(lower), arr(upper), n, ord, 1.0)
    assert h
    calls = 0
    try:
        for _ in range(100000):
            k = lib.nb_search_ask(h, None, 0)
            if k == 0:
                break
            pts = (ctypes.c_double * (k * n))()
            assert lib.nb_search_ask(h, pts, k) == k
            order = lib.nb_search_order(h)
            values = []
            for i in range(k):
                calls += 1
                values.append(f([pts[i * n + j] for j in range(n)], order, calls))
            assert lib.nb_search_tell(h, arr(values), k) == 0
        else:
            raise AssertionError("the search did not end")
        x = (ctypes.c_double * n)()
        failed = ctypes.c_int32(-1)
        evals = ctypes.c_uint32(0)
        found = lib.nb_search_result(h, x, ctypes.byref(failed), ctypes.byref(evals))
        assert evals.value == calls
        return found, list(x), failed.value, lib.nb_search_order(h)
    finally:
        lib.nb_search_free(h)


def bowl(x, *_):
    return (x[0] - 0.3) ** 2 + 0.01 * (x[1] - 4.0) ** 2


def test_search_finds_an_interior_minimum():
    found, x, failed, order = run_search([0.5, 2.0], 1, bowl)
    assert found == 1 and failed == 0 and order == 1
    assert x[0] == pytest.approx(0.3, rel=1e-4) and x[1] == pytest.approx(4.0, rel=1e-4)


def test_search_retries_at_order_one_after_a_rejected_fit():
    # rejected from the fifth fit on at the raised order (nebula's `second <
    # -1` error); the order-one pass is clean
    found, x, failed, order = run_search(
        [0.5, 2.0], 3, lambda x, order, calls: math.inf if order > 1 and calls >= 5 else bowl(x))
    assert order == 1 and found == 1 and failed == 0
    assert x[0] == pytest.approx(0.3, rel=1e-4)


def test_search_abandons_a_non_finite_order_one_pass():
    found, _, _, _ = run_search([0.5, 2.0], 1, lambda x, order, calls: math.nan if calls == 7 else bowl(x))
    assert found == 0


def test_search_reports_a_roundoff_limited_bobyqa_as_failed():
    # the box and start of the bobyqa_roundoff trace, which nloptr ends at -4:
    # the point is kept and the gene records -50
    found, x, failed, _ = run_search([0.0, 0.0], 1, lambda x, *_: (x[0] + x[1] - 1.0) ** 2,
                                     lower=[-2.0, -2.0], upper=[2.0, 2.0])
    assert found == 1 and failed == 1
    assert abs(x[0] + x[1] - 1.0) <= 1e-6


def test_one_component_search_keeps_a_genuine_bound():
    found, x, failed, _ = run_search([0.5], 1, lambda x, *_: x[0])
    assert found == 1 and failed == 0 and x[0] == 1e-4


def test_one_component_search_abandons_a_non_finite_start():
    found, _, _, _ = run_search([0.5], 1, lambda x, order, calls: math.inf if calls == 1 else x[0])
    assert found == 0


def test_search_refuses_a_wrong_number_of_values_and_bad_arguments():
    h = lib.nb_search_new(arr([0.5, 2.0]), arr([1e-4, 1e-4]), arr([10.0, 1000.0]), 2, 1, 1.0)
    try:
        assert lib.nb_search_ask(h, None, 0) == 1
        assert _ffi.STATUS_NAMES[lib.nb_search_tell(h, arr([1.0, 2.0]), 2)] == "LengthMismatch"
        assert lib.nb_search_result(h, None, None, None) == -1  # still running
    finally:
        lib.nb_search_free(h)
    assert not lib.nb_search_new(arr([0.5, 2.0]), arr([1e-4, 1e-4]), arr([10.0, 1000.0]), 3, 1, 1.0)
    assert not lib.nb_search_new(arr([0.5, 2.0]), arr([1e-4, 1e-4]), arr([10.0, 1000.0]), 2, 4, 1.0)
    assert not lib.nb_search_new(arr([math.nan, 2.0]), arr([1e-4, 1e-4]), arr([10.0, 1000.0]), 2, 1, 1.0)


def test_bobyqa_stops_when_its_evaluation_budget_runs_out():
    h = lib.nb_bobyqa_new(arr([0.5, 2.0]), arr([1e-4, 1e-4]), arr([10.0, 1000.0]), 2, 1e-6, 7)
    x = (ctypes.c_double * 2)()
    calls = 0
    while lib.nb_bobyqa_ask(h, x):
        calls += 1
        lib.nb_bobyqa_tell(h, bowl(list(x)))
        assert calls <= 7
    f = ctypes.c_double()
    evals = ctypes.c_uint32()
    status = lib.nb_bobyqa_result(h, x, ctypes.byref(f), ctypes.byref(evals))
    lib.nb_bobyqa_free(h)
    assert status == 5 and evals.value == 7 and calls == 7  # NLOPT_MAXEVAL_REACHED
    assert math.isfinite(f.value)


def small_inputs():
    rng = np.random.default_rng(5)
    n_cells, n_genes = 40, 3
    dense = rng.poisson(1.0, (n_genes, n_cells)).astype(float)
    indptr, indices, data = [0], [], []
    for row in dense:
        nz = np.flatnonzero(row)
        indices += nz.tolist()
        data += row[nz].tolist()
        indptr.append(len(data))
    csr = (np.array(indptr, np.uint32), np.array(indices, np.uint32), np.array(data), (n_genes, n_cells))
    subject = np.repeat(np.arange(4), 10)
    design = np.column_stack([np.ones(n_cells), rng.standard_normal(n_cells)])
    return csr, subject, design


def variant_of(fn):
    with pytest.raises(NebulaError) as e:
        fn()
    return e.value.variant


@pytest.mark.parametrize("bad", [math.nan, math.inf, -math.inf])
def test_non_finite_counts_design_and_offsets_are_refused(bad):
    csr, subject, design = small_inputs()
    indptr, indices, data, shape = csr
    poisoned = data.copy()
    poisoned[len(poisoned) // 2] = bad
    assert variant_of(lambda: nebula_sparse_cuda((indptr, indices, poisoned, shape), subject, design, 2)) \
        == "InvalidArgument"
    d = design.copy()
    d[7, 1] = bad
    assert variant_of(lambda: nebula_sparse_cuda(csr, subject, d, 2)) == "InvalidArgument"
    off = np.ones(40)
    off[3] = bad
    assert variant_of(lambda: nebula_sparse_cuda(csr, subject, design, 2, offset=off)) == "MustBePositive"
