"""ctypes access to the product's kernel-level entry nb_opt_pml_cuda (GPU only)."""
import ctypes

import numpy as np

from edge_rs_b200 import _ffi
from edge_rs_b200.api import NebulaError

_SIG = False


def _lib():
    global _SIG
    lib = _ffi.product_library()
    if not _SIG:
        lib.nb_opt_pml_cuda.restype = ctypes.c_int32
        _SIG = True
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def opt_pml_batch(design, offset, n_beta, counts, cells, subject_start, subject_total, beta_init, subject, cell,
                  ord=None, reml=False, eps=1e-6):
    """Runs len(subject) device inner fits of one gene; returns a list of dicts."""
    design = np.ascontiguousarray(design, np.float64)
    offset = np.ascontiguousarray(offset, np.float64)
    counts = np.ascontiguousarray(counts, np.float64)
    cells = np.ascontiguousarray(cells, np.uint32)
    ss = np.ascontiguousarray(subject_start, np.uint64)
    tot = np.ascontiguousarray(subject_total, np.float64)
    subject = np.atleast_1d(np.asarray(subject, np.float64))
    n_req = subject.size
    cell = np.ascontiguousarray(np.broadcast_to(np.asarray(cell, np.float64), (n_req,)))
    b0 = np.ascontiguousarray(np.broadcast_to(np.asarray(beta_init, np.float64), (n_req, n_beta)))
    ordv = np.ascontiguousarray(np.broadcast_to(np.asarray(1 if ord is None else ord, np.int32), (n_req,)))
    k = ss.size - 1
    beta = np.zeros((n_req, n_beta))
    info = np.zeros((n_req, n_beta * n_beta))
    sc = np.zeros((n_req, 4))
    ints = np.zeros((n_req, 4), np.int32)
    err = ctypes.create_string_buffer(256)
    rc = _lib().nb_opt_pml_cuda(_p(design), _p(offset), ctypes.c_uint64(offset.size), ctypes.c_uint32(n_beta),
                                _p(counts), _p(cells), ctypes.c_uint64(counts.size), _p(ss), ctypes.c_uint32(k),
                                _p(tot), ctypes.c_uint32(n_req), _p(b0), _p(subject), _p(cell), _p(ordv),
                                ctypes.c_int32(int(reml)), ctypes.c_double(eps), _p(beta), _p(info), _p(sc),
                                _p(ints), err, ctypes.c_size_t(len(err)))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return [dict(beta=beta[q], information=info[q], log_likelihood=sc[q, 0], log_likelihood_prev=sc[q, 1],
                 log_det=sc[q, 2], second_order=sc[q, 3], status=int(ints[q, 0]), iterations=int(ints[q, 1]),
                 backtracks=int(ints[q, 2]), sweeps=int(ints[q, 3])) for q in range(n_req)]
