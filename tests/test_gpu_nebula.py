"""nebula_sparse_cuda end to end against the oracle and the R goldens.

Against the FP64 oracle on the same inputs: beta, sigma^2 and phi to
relative 1e-6 and Wald log p-values to 1e-4 (the bar the path is held to);
against R's nebula output, the reference's own gates (tests/e2e_nebula.rs).
"""
import numpy as np
import pytest

import golden_io as gio
import oracle_ffi as of
from edge_rs_b200 import NebulaParams, glm_sc_test, nebula_sparse_cuda, workloads

pytestmark = pytest.mark.gpu

REL_PARAM = 1e-6   # beta, sigma^2, phi against the oracle
REL_LOGP = 1e-4    # log p-value against the oracle


def compare_to_oracle(dev, ref, label):
    assert np.array_equal(dev.gene_index, ref.gene_index), label
    # the device path and the oracle share their summation trees and exp/log,
    # so they agree bit for bit; the tolerances below are the stated bar
    for key in ("coefficients", "se", "covariance", "subject_overdispersion", "cell_overdispersion",
                "convergence"):
        a, b = getattr(dev, key), getattr(ref, key)
        same = np.array_equal(a, b, equal_nan=True)
        assert same, f"{label}: {key} not bit-identical (max diff {np.nanmax(np.abs(a - b)):.3e})"
    for key in ("coefficients", "subject_overdispersion", "cell_overdispersion"):
        ok, worst = gio.close(getattr(dev, key), getattr(ref, key), REL_PARAM, 1e-9)
        assert ok, f"{label}: {key} off by {worst:.2e}"
    ok, worst = gio.close(dev.se, ref.se, 1e-5, 1e-12)
    assert ok, f"{label}: se off by {worst:.2e}"
    for coef in range(1, dev.n_coef):
        a = glm_sc_test(dev.coefficients, dev.covariance, coef=coef).log_p_value
        b = glm_sc_test(ref.coefficients, ref.covariance, coef=coef).log_p_value
        ok, worst = gio.close(a, b, REL_LOGP, 1e-6)
        assert ok, f"{label}: log p of coefficient {coef} off by {worst:.2e}"


def test_eight_gene_golden_on_the_device():
    d = gio.load_eight_gene()
    w = gio.expected_eight_gene()
    params = NebulaParams(cutoff_cell=0.0)
    dev = nebula_sparse_cuda(d["csr"], d["subject"], d["design"], 3, d["offset"], params)
    ref, _ = of.nebula_sparse(d["csr"], d["subject"], d["design"], 3, d["offset"], params, threads=4)
    compare_to_oracle(dev, ref, "8-gene")
    assert gio.close(dev.coefficients, w["coef"], 5e-6)[0]
    assert gio.close(dev.subject_overdispersion, w["subject"], 1e-5)[0]
    assert gio.close(dev.cell_overdispersion, w["cell"], 1e-5)[0]
    assert gio.close(dev.covariance, w["cov"], 1e-5)[0]
    for coef in (1, 2):
        p = glm_sc_test(dev.coefficients, dev.covariance, coef=coef).p_value
        assert gio.close(p, w["p"][:, coef], 1e-4)[0]


@pytest.mark.parametrize("tag", gio.inline()["e2e_hl"])
def test_hl_datasets_match_the_oracle_and_r(tag):
    d = gio.load_e2e(tag)
    params = NebulaParams(method=d["method"])
    dev = nebula_sparse_cuda(d["csr"], d["subject"], d["design"], d["n_coef"], d["offset"], params)
    ref, _ = of.nebula_sparse(d["csr"], d["subject"], d["design"], d["n_coef"], d["offset"], params, threads=4)
    compare_to_oracle(dev, ref, tag)
    w = gio.expected_e2e(tag, d["n_coef"])
    loose = tag == "sc_high"
    assert gio.close(dev.coefficients, w["coef"], 3e-4 if loose else 3e-5, 1e-9)[0]
    assert gio.close(dev.subject_overdispersion, w["subject"], 2e-3 if loose else 2e-4, 1e-6)[0]


@pytest.mark.parametrize("tag", [t for t in gio.inline()["e2e_ln"] if gio.E2E[t][2] <= 8])
def test_ln_datasets_match_the_oracle(tag):
    d = gio.load_e2e(tag)
    params = NebulaParams(method=d["method"])
    dev = nebula_sparse_cuda(d["csr"], d["subject"], d["design"], d["n_coef"], d["offset"], params)
    ref, _ = of.nebula_sparse(d["csr"], d["subject"], d["design"], d["n_coef"], d["offset"], params, threads=4)
    compare_to_oracle(dev, ref, tag)


@pytest.mark.parametrize("name,genes,cells,k", [("c0", 24, 5000, 10), ("c1", 12, 20000, 20), ("c2", 12, 8000, 32)])
def test_synthetic_configs_match_the_oracle(name, genes, cells, k):
    w = workloads.make(name, seed=11, n_genes=genes, n_cells=cells, n_subjects=k)
    params = NebulaParams(method="HL")
    dev = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params)
    ref, _ = of.nebula_sparse(w.csr, w.subject, w.design, w.n_coef, w.offset, params, threads=8)
    compare_to_oracle(dev, ref, name)
    assert dev.stats["requests"] > 0 and dev.stats["gpu_launches"] > 0


@pytest.mark.parametrize("name,genes", [("c1", 6), ("c2", 10), ("c3", 5), ("c4", 6)])
def test_configs_at_full_size_match_the_oracle(name, genes):
    """A few genes of each benchmark configuration at its stated cell and
    subject counts: c1 100,000 cells x 20 subjects (4 columns), c2 50,000 x 64
    of 100-5,000 cells (8 columns, five varying within subjects, nnz over
    three decades), c3 200,000 x 40 (8 columns), c4 100,000 x 100 (4 columns)."""
    w = workloads.make(name, seed=21, n_genes=genes)
    assert w.n_cells == workloads.CONFIGS[name]["n_cells"]
    params = NebulaParams(method="HL")
    dev = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params)
    ref, _ = of.nebula_sparse(w.csr, w.subject, w.design, w.n_coef, w.offset, params, threads=8)
    compare_to_oracle(dev, ref, name)


def test_results_are_reproducible_run_to_run():
    w = workloads.make("c1", seed=5, n_genes=8, n_cells=10000, n_subjects=12)
    params = NebulaParams(method="HL")
    a = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params)
    b = nebula_sparse_cuda(w.csr, w.subject, w.design, w.n_coef, w.offset, params)
    assert np.array_equal(a.coefficients, b.coefficients)
    assert np.array_equal(a.subject_overdispersion, b.subject_overdispersion)
