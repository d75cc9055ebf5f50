"""Zero-count tables on the device: the fit kernel's tabled sweep (the loose
cells visited one by one, each tabled group looked up per subject) against the
FP64 oracle's, which evaluates the same tables in the same order, so the two
agree bit for bit. Both a fully tabled design and one that leaves some cells
loose are checked, at the Laplace orders that use the higher sums."""
import numpy as np
import pytest

import oracle_ffi as of
from device_ffi import opt_pml_batch
from test_zero_tables import categorical_gene, groups

pytestmark = pytest.mark.gpu

POINTS = [(0.3, 0.05, 3), (0.8, 2.0, 2), (0.05, 40.0, 1), (1.2, 0.5, 3)]


def with_loose_cells(design):
    """Every 37th cell gets its own value in the cell-level column, leaving it
    in a group too small to table."""
    d = design.copy()
    d[::37, 2] = 0.5
    return d


@pytest.mark.parametrize("loose", [False, True])
def test_device_tabled_fit_matches_the_oracle_bitwise(loose):
    design, offset, counts, cells, starts, total = categorical_gene()
    if loose:
        design = with_loose_cells(design)
    g, _, loose_cells = groups(design, offset, starts)
    assert g == 6 and (loose_cells.size > 0) == loose
    start = np.array([-1.5, 0.2, 0.1])
    dev = opt_pml_batch(design.reshape(-1), offset, 3, counts, cells, starts, total, start,
                        [p[0] for p in POINTS], [p[1] for p in POINTS], ord=[p[2] for p in POINTS], reml=True)
    for q, (s, c, o) in enumerate(POINTS):
        ref = of.opt_pml(design.reshape(-1), offset, 3, counts, cells, starts, total, start, s, c, reml=True, ord=o)
        d = dev[q]
        assert d["status"] == 0
        assert d["iterations"] == ref["iterations"] and d["backtracks"] == ref["backtracks"], q
        assert np.array_equal(d["beta"], ref["beta"]), q
        assert np.array_equal(d["information"], ref["information"]), q
        for key in ("log_likelihood", "log_likelihood_prev", "log_det", "second_order"):
            assert d[key] == ref[key], (q, key)


def test_device_tabled_fit_differs_from_dense_only_in_rounding():
    """The same fits with the tables switched off in the oracle: the device's
    tabled results stay within the reference's tabled-versus-dense bounds."""
    design, offset, counts, cells, starts, total = categorical_gene()
    start = np.array([-1.5, 0.2, 0.1])
    dev = opt_pml_batch(design.reshape(-1), offset, 3, counts, cells, starts, total, start,
                        [p[0] for p in POINTS], [p[1] for p in POINTS], ord=[p[2] for p in POINTS], reml=True)
    for q, (s, c, o) in enumerate(POINTS):
        dense = of.opt_pml(design.reshape(-1), offset, 3, counts, cells, starts, total, start, s, c, reml=True,
                           ord=o, tabled=False)
        assert dev[q]["log_likelihood"] == pytest.approx(dense["log_likelihood"], rel=1e-13)
        assert dev[q]["log_det"] == pytest.approx(dense["log_det"], rel=1e-12)
        np.testing.assert_allclose(dev[q]["beta"], dense["beta"], rtol=1e-6)


def test_categorical_fit_uses_the_tables_and_matches_the_dense_sweep():
    """nebula_sparse_cuda on a categorical design (intercept and a
    subject-level binary): one tabled group per subject, and the fits agree
    with the same call sweeping every cell within the search's resolution
    (the objective differs in its last digits, so BOBYQA may stop at a
    different point within its final radius)."""
    from edge_rs_b200 import NebulaParams, nebula_sparse_cuda, workloads
    w = workloads.make("c0", seed=3, n_genes=24, n_cells=5000, n_subjects=10)
    params = NebulaParams(method="HL")
    tabled = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params)
    dense = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params, dense_sweep=True)
    assert tabled.stats["zero_groups"] == 10 and dense.stats["zero_groups"] == 0
    assert tabled.stats["cell_visits"] < 0.5 * dense.stats["cell_visits"]
    assert np.array_equal(tabled.gene_index, dense.gene_index)
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1e-12)
    assert np.median(rel(tabled.coefficients, dense.coefficients)) < 1e-6
    assert np.median(rel(tabled.subject_overdispersion, dense.subject_overdispersion)) < 1e-4
    assert np.median(rel(tabled.cell_overdispersion, dense.cell_overdispersion)) < 1e-4


def test_continuous_design_builds_no_tables():
    from edge_rs_b200 import NebulaParams, nebula_sparse_cuda, workloads
    w = workloads.make("c1", seed=3, n_genes=8, n_cells=4000, n_subjects=8)
    fit = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"))
    assert fit.stats["zero_groups"] == 0
