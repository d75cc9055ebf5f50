"""B200-native NEBULA-HL stage two, a drop-in for edge-rs's nebula_sparse.

The product is libnebula_b200.so (C-ABI in include/nebula_cuda.h): host C++
for stage one, the stage-two search and stage three's finish, and CUDA
kernels for sm_100a that run every penalised NB-gamma inner fit. This module
is the thin Python mirror of the reference's Rust interface.
"""
from .api import (NebulaError, NebulaFit, NebulaParams, ScTestResult, Session, glm_sc_test, glm_sc_test_cuda, mlp_gradient,
                  mlp_init, mlp_predict, mlp_train, nebula_sparse_cuda, opt_pml_cuda)

__all__ = ["NebulaError", "NebulaFit", "NebulaParams", "ScTestResult", "Session", "glm_sc_test", "glm_sc_test_cuda",
           "mlp_gradient", "mlp_init", "mlp_predict", "mlp_train", "nebula_sparse_cuda", "opt_pml_cuda"]
