"""The C-ABI library loads on a CPU-only host, exports every symbol the header
declares, and rejects malformed inputs before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from edge_rs_b200 import NebulaError, NebulaParams, _ffi, nebula_sparse_cuda

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "nebula_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(n[a-z_]+)\s*\(", text)) - {"nb_status"})


def test_header_declares_the_drop_in():
    names = declared_functions()
    for required in ("nebula_sparse_cuda", "nebula_sparse_cuda_ex", "nb_glm_sc_test", "nb_opt_pml_cuda"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_ffi.PRODUCT_LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_params_default_are_the_r_package_defaults():
    lib = _ffi.product_library()
    p = _ffi.NbParams()
    lib.nb_params_default(ctypes.byref(p))
    assert (p.min_subject, p.min_cell, p.max_subject, p.max_cell) == (1e-4, 1e-4, 10.0, 1000.0)
    assert p.method == _ffi.NB_METHOD_LN and p.cutoff_cell == 20.0 and p.kappa == 800.0
    assert p.cpc == 0.005 and p.mincp == 5 and p.min_subjects == 0 and p.reml == 0 and p.eps == 1e-6


def small_inputs(n_coef=2):
    rng = np.random.default_rng(3)
    n_cells, n_genes = 40, 3
    dense = rng.poisson(1.0, (n_genes, n_cells)).astype(float)
    indptr = [0]
    indices, data = [], []
    for row in dense:
        nz = np.flatnonzero(row)
        indices += nz.tolist()
        data += row[nz].tolist()
        indptr.append(len(data))
    csr = (np.array(indptr, np.uint32), np.array(indices, np.uint32), np.array(data), (n_genes, n_cells))
    subject = np.repeat(np.arange(4), 10)
    design = np.column_stack([np.ones(n_cells)] + [rng.standard_normal(n_cells) for _ in range(n_coef - 1)])
    return csr, subject, design


def code_of(fn):
    with pytest.raises(NebulaError) as e:
        fn()
    return e.value.variant


def test_rejects_more_than_eight_columns_like_the_device_path():
    csr, subject, design = small_inputs(9)
    assert code_of(lambda: nebula_sparse_cuda(csr, subject, design, 9)) == "Unsupported"


def test_rejects_malformed_inputs_before_any_device_work():
    csr, subject, design = small_inputs()
    indptr, indices, data, shape = csr
    bad = (indptr, indices.copy(), data, shape)
    bad[1][0] = 999
    assert code_of(lambda: nebula_sparse_cuda(bad, subject, design, 2)) == "MalformedSparse"
    neg = (indptr, indices, -data, shape)
    assert code_of(lambda: nebula_sparse_cuda(neg, subject, design, 2)) == "InvalidArgument"
    split = subject.copy()
    split[:5] = 3
    assert code_of(lambda: nebula_sparse_cuda(csr, split, design, 2)) == "SubjectsNotContiguous"
    one = np.zeros_like(subject)
    assert code_of(lambda: nebula_sparse_cuda(csr, one, design, 2)) == "TooFewSubjects"
    no_icpt = design.copy()
    no_icpt[:, 0] = np.arange(40.0)
    assert code_of(lambda: nebula_sparse_cuda(csr, subject, no_icpt, 2)) == "MissingIntercept"
    assert code_of(lambda: nebula_sparse_cuda(csr, subject, design, 2, offset=np.zeros(40))) == "MustBePositive"
    p = NebulaParams(min=(0.0, 1e-4))
    assert code_of(lambda: nebula_sparse_cuda(csr, subject, design, 2, params=p)) == "MustBePositive"
    p = NebulaParams(cpc=1e9)
    assert code_of(lambda: nebula_sparse_cuda(csr, subject, design, 2, params=p)) == "NoGenesAfterFiltering"
    empty = (np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0), (0, 40))
    assert code_of(lambda: nebula_sparse_cuda(empty, subject, design, 2)) == "EmptyCounts"
