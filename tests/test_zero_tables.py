"""Zero-count tables (edge_rs_b200/csrc/host/zero_tables.hpp, the reference's
src/sc/zeros.rs) on the CPU, through the oracle library that shares them with
the device path.

- The tables of a group match its sums computed directly, over the whole
  range of s and across the ends where the closed forms take over (the bounds
  of zeros.rs:493-592).
- Grouping: a continuous cell-level column builds no tables; a categorical
  design tables its large groups and leaves the small ones loose.
- An inner fit with the tables matches the same fit sweeping every cell, to
  the tolerances the reference holds its tabled fit to (pml.rs:2926-2965).
"""
import ctypes
import math

import numpy as np
import pytest

import oracle_ffi as of


def _lib():
    lib = of.lib()
    lib.oracle_zero_eval.restype = ctypes.c_int32
    lib.oracle_zero_groups.restype = ctypes.c_int32
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def table_sums(log_o, s, start=0, count=6):
    log_o = np.ascontiguousarray(log_o, np.float64)
    s = np.ascontiguousarray(np.atleast_1d(s), np.float64)
    out = np.zeros((s.size, count))
    rng = np.zeros(2)
    rc = _lib().oracle_zero_eval(_p(log_o), ctypes.c_uint64(log_o.size), _p(s), ctypes.c_uint64(s.size),
                                 ctypes.c_int32(start), ctypes.c_int32(count), _p(out), _p(rng))
    assert rc == 0
    return out, rng


def direct_sums(log_o, s):
    """The six sums at s, each an exactly rounded sum (math.fsum)."""
    v = np.exp(s + np.asarray(log_o))
    w = 1.0 / (1.0 + v)
    u = v * w
    uw = u * w
    terms = [np.log1p(v), u, uw, uw * (w - u), uw * (w * w - 4 * u * w + u * u),
             uw * (w ** 3 - 11 * w * w * u + 11 * w * u * u - u ** 3)]
    return np.array([math.fsum(t) for t in terms])


def offsets(n, seed):
    """Log offsets spread like library sizes over two orders of magnitude."""
    return np.random.default_rng(seed).uniform(6.0, 10.6, n)


def relative_errors(got, want):
    # C, D and E change sign and are judged against B, the scale they are stored at
    scale = np.array([abs(want[0]), abs(want[1]), abs(want[2]), want[2], want[2], want[2]])
    return np.abs(got - want) / scale


def test_tables_match_direct_sums_over_the_whole_range():
    log_o = offsets(500, 7)
    _, (s_lo, s_hi) = table_sums(log_o, 0.0)
    s = np.arange(s_lo - 5.0, s_hi + 5.0, 0.0137)
    got, _ = table_sums(log_o, s)
    worst = np.zeros(6)
    for i in range(s.size):
        worst = np.maximum(worst, relative_errors(got[i], direct_sums(log_o, s[i])))
    assert np.all(worst < 1e-13), worst


def test_tables_are_continuous_across_their_ends():
    log_o = offsets(300, 11)
    _, (s_lo, s_hi) = table_sums(log_o, 0.0)
    for edge in (s_lo, s_hi):
        for s in (edge - 1e-9, edge, edge + 1e-9):
            got, _ = table_sums(log_o, s)
            assert np.all(relative_errors(got[0], direct_sums(log_o, s)) <= 1e-12), (edge, s)


def test_tables_handle_infinite_and_nan_arguments():
    log_o = offsets(100, 13)
    low, _ = table_sums(log_o, -np.inf)
    assert np.all(low == 0.0)
    high, _ = table_sums(log_o, np.inf, 0, 3)
    assert high[0, 0] == np.inf and high[0, 1] == log_o.size
    nan, _ = table_sums(log_o, np.nan)
    assert np.all(np.isnan(nan))


def groups(design, log_o, starts):
    design = np.ascontiguousarray(design, np.float64)
    n_coef = design.shape[1]
    n = design.shape[0]
    rows = np.zeros(n, np.int64)
    loose = np.zeros(n, np.uint32)
    n_loose = ctypes.c_uint64()
    ss = np.ascontiguousarray(starts, np.uint64)
    g = _lib().oracle_zero_groups(_p(design), _p(np.ascontiguousarray(log_o, np.float64)), _p(ss),
                                  ctypes.c_uint32(ss.size - 1), ctypes.c_uint32(n_coef), _p(rows), _p(loose),
                                  ctypes.byref(n_loose))
    return g, rows[:max(g, 0)], loose[:n_loose.value]


def test_build_skips_a_continuous_design():
    n = 400
    rng = np.random.default_rng(9)
    design = np.column_stack([np.ones(n), rng.uniform(-1, 1, n)])
    g, _, _ = groups(design, offsets(n, 3), [0, 200, 400])
    assert g == -1


def test_build_groups_a_categorical_design():
    n = 400
    r = np.arange(n)
    design = np.column_stack([np.ones(n), r % 3, np.where(r % 50 == 0, 0.5, 0.0)])
    g, rows, loose = groups(design, offsets(n, 3), [0, 200, 400])
    assert g == 6  # three levels in each of two subjects
    # the rows with the odd third column are too few to table
    assert loose.tolist() == [0, 50, 100, 150, 200, 250, 300, 350]
    assert rows.tolist() == [1, 2, 3, 201, 202, 203]


def categorical_gene(seed=11):
    """Three subjects of 400 cells; intercept, a subject-level binary and a
    cell-level binary (drawn with probability 0.4); offsets uniform on
    (-2.3, 2.3); a count of 1 to 5 with probability 0.1 (0.15 where the cell
    binary is set)."""
    rng = np.random.default_rng(seed)
    n = 1200
    s = np.arange(n) // 400
    kind = (rng.random(n) < 0.4).astype(float)
    design = np.column_stack([np.ones(n), (s % 2).astype(float), kind])
    offset = rng.uniform(-2.3, 2.3, n)
    positive = rng.random(n) < 0.1 + 0.05 * kind
    cells = np.flatnonzero(positive).astype(np.uint32)
    counts = rng.integers(1, 6, cells.size).astype(float)
    total = np.bincount(s[cells], weights=counts, minlength=3)
    starts = np.array([0, 400, 800, 1200], np.uint64)
    return design, offset, counts, cells, starts, total


@pytest.mark.parametrize("subject,cell", [(0.3, 0.05), (0.8, 2.0), (0.05, 40.0)])
def test_tabled_inner_fit_matches_the_dense_sweep(subject, cell):
    """Every Newton iterate of the tabled fit matches the dense one to 1e-11
    (the tables' sums agree to ~1e-14), and the converged fits agree to the
    reference's tolerances on the log-likelihood, the log-determinant and the
    information. The final step is judged by the Newton tolerance instead: at
    the optimum the likelihood change is rounding-level, and its sign, which
    decides whether the last step is halved once more, can differ between the
    two (it does at (0.05, 40) on this draw: one backtrack against none)."""
    design, offset, counts, cells, starts, total = categorical_gene()
    g, _, loose = groups(design, offset, starts)
    assert g == 6 and loose.size == 0
    start = np.array([-1.5, 0.2, 0.1])
    run = lambda tabled, max_iter=50: of.opt_pml(design.reshape(-1), offset, 3, counts, cells, starts, total, start,
                                                 subject, cell, reml=True, ord=3, max_iter=max_iter, tabled=tabled)
    dense, tabled = run(False), run(True)
    assert dense["iterations"] == tabled["iterations"]
    for steps in range(1, dense["iterations"]):
        np.testing.assert_allclose(run(True, steps)["beta"], run(False, steps)["beta"], rtol=1e-11)
    np.testing.assert_allclose(tabled["beta"], dense["beta"], rtol=1e-6)
    np.testing.assert_allclose(tabled["information"], dense["information"], rtol=1e-11)
    assert tabled["log_likelihood"] == pytest.approx(dense["log_likelihood"], rel=1e-13)
    assert tabled["log_det"] == pytest.approx(dense["log_det"], rel=1e-12)
    assert tabled["second_order"] == pytest.approx(dense["second_order"], rel=1e-8)
