"""The Hessian contraction S_r = sum_c w_rc x_c x_c' (nb_contract_krx_cuda) in
its four arithmetics against an FP64 numpy product of the same inputs: FP64
on CUDA cores to 1e-12, FP32 on CUDA cores and split BF16 on the tensor cores
(tcgen05.mma, three BF16 products, FP32 accumulation) to 1e-5, TF32 on the
tensor cores to 5e-3, each relative to the largest entry of the request's
S. Ragged sizes: cells not a multiple of the K tile, fewer than 128
requests, fewer than 8 columns."""
import numpy as np
import pytest

from edge_rs_b200.api import contract_krx_cuda

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-5, 2: 5e-3, 3: 1e-5}


@pytest.mark.parametrize("n_cells,n_coef,n_req", [(1000, 2, 3), (20011, 8, 128), (65536, 4, 37)])
def test_contraction_variants_against_fp64(n_cells, n_coef, n_req):
    import torch
    rng = np.random.default_rng(n_cells)
    x = rng.standard_normal((n_cells, n_coef))
    x[:, 0] = 1.0
    w = np.exp(rng.normal(-2.0, 1.5, (n_req, n_cells)))  # positive weights over decades, as a sweep's
    pairs = [(a, b) for b in range(n_coef) for a in range(b + 1)]
    want = np.stack([w @ (x[:, a] * x[:, b]) for a, b in pairs], axis=1)
    dx = torch.from_numpy(x).cuda()
    dw = torch.from_numpy(w).cuda()
    scale = np.abs(want).max(axis=1, keepdims=True)
    for variant, tol in TOL.items():
        got, ms, ms_total = contract_krx_cuda(variant, dx, dw)
        err = np.abs(got.cpu().numpy() - want) / scale
        assert err.max() <= tol, (variant, err.max())
        assert 0.0 < ms <= ms_total
