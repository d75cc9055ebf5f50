"""glm_sc_test reproduces nebula's Wald p-values (src/sc/nebula.rs:2502-2537, test.rs:214-382)."""
import numpy as np

import golden_io as gio
import oracle_ffi as of
from edge_rs_b200 import NebulaParams, glm_sc_test


def test_wald_reproduces_the_r_p_values_from_the_oracle_fit():
    d = gio.load_eight_gene()
    w = gio.expected_eight_gene()
    fit, _ = of.nebula_sparse(d["csr"], d["subject"], d["design"], 3, d["offset"], NebulaParams(cutoff_cell=0.0),
                              threads=2)
    for coef in (1, 2):
        res = glm_sc_test(fit.coefficients, fit.covariance, coef=coef)
        ok, worst = gio.close(res.p_value, w["p"][:, coef], 1e-4)
        assert ok, worst
        assert np.allclose(np.exp(res.log_p_value), res.p_value, rtol=1e-12, atol=0)


def test_wald_contrast_uses_the_full_covariance_and_bh():
    beta = np.array([[1.0, 2.0], [0.0, 0.5], [3.0, -1.0]])
    cov = np.array([[1.0, 0.5, 4.0], [1.0, 0.0, 1.0], [2.0, -1.0, 2.0]])  # packed V11, V12, V22
    res = glm_sc_test(beta, cov, contrast=np.array([1.0, -1.0]))
    var = cov[:, 0] + cov[:, 2] - 2 * cov[:, 1]
    assert np.allclose(res.log_fc, beta[:, 0] - beta[:, 1])
    assert np.allclose(res.se, np.sqrt(var))
    from math import erfc, sqrt
    p = np.array([erfc(abs(z) / sqrt(2)) for z in res.z])
    assert np.allclose(res.p_value, p, rtol=1e-14)
    order = np.argsort(-p, kind="stable")
    running, bh = np.inf, np.zeros(3)
    for j, i in enumerate(order):
        running = min(running, 3 / (3 - j) * p[i])
        bh[i] = min(running, 1.0)
    assert np.allclose(res.fdr, bh)


def test_wald_log_p_stays_finite_where_p_underflows():
    beta = np.array([[0.0, 60.0]])
    cov = np.array([[1.0, 0.0, 1.0]])
    res = glm_sc_test(beta, cov, coef=1)
    assert res.p_value[0] == 0.0
    # log erfc(60/sqrt(2)) = -1800 - log(60/sqrt(2) * sqrt(pi)) + log(1 - 1/3600 + ...)
    x = 60 / np.sqrt(2)
    want = -x * x - np.log(x * np.sqrt(np.pi)) + np.log(1 - 1 / (2 * x * x) + 3 / (4 * x ** 4))
    assert abs(res.log_p_value[0] - want) < 1e-9
