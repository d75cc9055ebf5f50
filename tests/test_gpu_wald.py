"""glm_sc_test on the device (nb_glm_sc_test_cuda) against the host
nb_glm_sc_test (src/sc/test.rs:96-200) on the same fits: the effect, its
standard error and z bit for bit (the same arithmetic in the same order),
p-values, log p-values and BH FDR to 1e-13 relative (CUDA's erfc and log
against the host's; log p also within 1e-14 absolute where p is near one), including p-values that underflow, ties and a
contrast."""
import numpy as np
import pytest

from edge_rs_b200 import glm_sc_test, glm_sc_test_cuda

pytestmark = pytest.mark.gpu


def random_fits(rng, n_genes, n_coef):
    beta = rng.normal(0.0, 1.0, (n_genes, n_coef))
    beta[: n_genes // 10, 1] *= 40.0        # z far in the tail: p underflows, log p does not
    beta[n_genes // 10: n_genes // 5, 1] = 0.0  # z = 0: p = 1, ties for BH
    packed = []
    for _ in range(n_genes):
        a = rng.normal(0.0, 0.3, (n_coef, n_coef))
        v = a @ a.T + 0.05 * np.eye(n_coef)
        packed.append([v[i, j] for j in range(n_coef) for i in range(j + 1)])
    return beta, np.array(packed)


def close(a, b, rel, eps=0.0):
    a, b = np.asarray(a), np.asarray(b)
    same = (a == b) | (np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b))) | (np.abs(a - b) <= eps)
    return bool(np.all(same)), float(np.max(np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)))


@pytest.mark.parametrize("n_genes,n_coef", [(1, 2), (4000, 4), (20000, 8)])
def test_device_wald_matches_the_host(n_genes, n_coef):
    import torch
    rng = np.random.default_rng(n_genes + n_coef)
    beta, cov = random_fits(rng, n_genes, n_coef)
    d_beta = torch.from_numpy(beta).cuda()
    d_cov = torch.from_numpy(cov).cuda()
    contrasts = [dict(coef=1), dict(contrast=np.r_[0.0, 1.0, -1.0, np.zeros(n_coef - 3)] if n_coef >= 3
                                    else np.array([1.0, -1.0]))]
    for kw in contrasts:
        host = glm_sc_test(beta, cov, **kw)
        dev = glm_sc_test_cuda(d_beta, d_cov, **kw)
        for key in ("log_fc", "se", "z"):
            assert np.array_equal(getattr(dev, key).cpu().numpy(), getattr(host, key)), key
        # log p near zero (p near one) inherits erfc's last-bit difference as
        # an absolute error of ~1e-16: 1e-14 absolute there
        for key, eps in (("p_value", 0.0), ("log_p_value", 1e-14), ("fdr", 0.0)):
            ok, worst = close(getattr(dev, key).cpu().numpy(), getattr(host, key), 1e-13, eps)
            assert ok, (key, worst)
    if n_genes > 1:
        res = glm_sc_test_cuda(d_beta, d_cov, coef=1)
        p = res.p_value.cpu().numpy()
        assert np.any(p == 0.0) and np.all(np.isfinite(res.log_p_value.cpu().numpy()))
