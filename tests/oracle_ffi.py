"""ctypes access to the oracle (oracle/liboracle.so), for tests and the CPU baseline only."""
import ctypes
import os

import numpy as np

from edge_rs_b200 import _ffi
from edge_rs_b200.api import NebulaError, NebulaParams, _as_csr, fit_from_arrays

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} is missing: build it with `make -C oracle`")
        _LIB = ctypes.CDLL(ORACLE_LIB)
        _LIB.oracle_opt_pml.restype = ctypes.c_int32
        _LIB.oracle_nebula_sparse.restype = ctypes.c_int32
        _LIB.oracle_pml_objective_gradient.restype = ctypes.c_double
        _LIB.oracle_min_eigenvalue.restype = ctypes.c_double
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def opt_pml(design, offset, n_beta, counts, cells, subject_start, subject_total, beta_init, subject, cell,
            reml=False, eps=1e-6, ord=1, max_iter=50, lognormal=False, log_w_init=None, tabled=True):
    """The oracle's opt_pml; with `tabled` the zero-count tables of the design
    and offsets are used where they apply (as the device path does), without
    it every cell is swept."""
    design = np.ascontiguousarray(design, np.float64)
    offset = np.ascontiguousarray(offset, np.float64)
    counts = np.ascontiguousarray(counts, np.float64)
    cells = np.ascontiguousarray(cells, np.uint32)
    ss = np.ascontiguousarray(subject_start, np.uint64)
    tot = np.ascontiguousarray(subject_total, np.float64)
    b0 = np.ascontiguousarray(beta_init, np.float64)
    lw0 = None if log_w_init is None else np.ascontiguousarray(log_w_init, np.float64)
    k = ss.size - 1
    beta = np.zeros(n_beta)
    log_w = np.zeros(k)
    info = np.zeros(n_beta * n_beta)
    sc = np.zeros(4)
    ints = np.zeros(4, np.int32)
    rc = lib().oracle_opt_pml(_p(design), _p(offset), ctypes.c_uint64(offset.size), ctypes.c_uint32(n_beta),
                              _p(counts), _p(cells), ctypes.c_uint64(counts.size), _p(ss), ctypes.c_uint32(k),
                              _p(tot), _p(b0), _p(lw0), ctypes.c_double(subject), ctypes.c_double(cell),
                              ctypes.c_int32(int(reml)), ctypes.c_double(eps), ctypes.c_int32(ord),
                              ctypes.c_int32(max_iter), ctypes.c_int32(int(lognormal)), ctypes.c_int32(int(tabled)),
                              _p(beta), _p(log_w),
                              _p(info), _p(sc), _p(ints))
    if rc != 0:
        raise NebulaError(rc, "opt_pml rejected its arguments")
    return dict(beta=beta, log_w=log_w, information=info, log_likelihood=sc[0], log_likelihood_prev=sc[1],
                log_det=sc[2], second_order=sc[3], convergence=int(ints[0]), iterations=int(ints[1]),
                backtracks=int(ints[2]), sweeps=int(ints[3]))


def nebula_sparse(counts, subject_id, design, n_coef, offset=None, params=None, threads=0):
    """The oracle's CPU nebula_sparse; returns (NebulaFit, work dict)."""
    csr = _as_csr(counts)
    n_genes, n_cells = int(csr.struct.n_genes), int(csr.struct.n_cells)
    subject = np.ascontiguousarray(subject_id, dtype=np.uint64)
    design = np.ascontiguousarray(design, dtype=np.float64).reshape(-1)
    off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float64)
    p = (params or NebulaParams()).to_c()
    out = _ffi.FitArrays(n_genes, n_coef)
    work = np.zeros(3, np.int64)
    err = ctypes.create_string_buffer(512)
    rc = lib().oracle_nebula_sparse(ctypes.byref(csr.struct), _p(subject), _p(design), ctypes.c_uint32(n_coef),
                                    _p(off), ctypes.byref(p), ctypes.c_int32(threads), ctypes.byref(out.struct),
                                    _p(work), err, ctypes.c_size_t(len(err)))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return fit_from_arrays(out, n_coef), dict(evaluations=int(work[0]), sweeps=int(work[1]), genes=int(work[2]))


def mlp_loss_grad(params, features, targets):
    """The FP64 oracle's loss and gradient of the warm-start network."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, 12)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
    g = np.zeros(p.size)
    loss = ctypes.c_double(0.0)
    lib().oracle_mlp_loss_grad(_p(p), _p(x), _p(t), ctypes.c_uint64(x.shape[0]), _p(g), ctypes.byref(loss))
    return loss.value, g


def mlp_predict(params, features):
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, 12)
    out = np.zeros((x.shape[0], 3))
    lib().oracle_mlp_predict(_p(p), _p(x), ctypes.c_uint64(x.shape[0]), _p(out))
    return out


_FG = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_uint32,
                       ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


def lbfgsb(fg, x0, lower, upper, memory=10, ftol=1e-6, pgtol=1e-5, max_iter=200, max_line_search=20):
    """The stage-one quasi-Newton (csrc/host/lbfgsb.cpp) on fg(x) -> (value,
    gradient). Returns (x, f, status, iterations, evaluations); a rejected
    argument raises NebulaError with the EdgeErrors code."""
    x0 = np.ascontiguousarray(x0, np.float64)
    lo = np.ascontiguousarray(lower, np.float64)
    hi = np.ascontiguousarray(upper, np.float64)
    n = x0.size

    def cb(x, m, grad, _ctx):
        xv = np.ctypeslib.as_array(x, shape=(m,)).copy()
        f, g = fg(xv)
        gv = np.ctypeslib.as_array(grad, shape=(m,))
        gv[:] = g
        return float(f)

    callback = _FG(cb)
    out = np.zeros(max(n, 1))
    f = ctypes.c_double(0.0)
    ints = np.zeros(3, np.int32)
    err = ctypes.create_string_buffer(256)
    rc = lib().oracle_lbfgsb(callback, None, _p(x0), ctypes.c_uint32(n), _p(lo), ctypes.c_uint32(lo.size), _p(hi),
                             ctypes.c_uint32(hi.size), ctypes.c_int32(memory), ctypes.c_double(ftol),
                             ctypes.c_double(pgtol), ctypes.c_int32(max_iter), ctypes.c_int32(max_line_search),
                             _p(out), ctypes.byref(f), _p(ints), err, ctypes.c_uint64(len(err)))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return out[:n], f.value, int(ints[0]), int(ints[1]), int(ints[2])


def lbfgsb_solve_dense(a, b):
    """solve_dense of the quasi-Newton; None when singular."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(b.size)
    rc = lib().oracle_lbfgsb_solve_dense(_p(a), _p(b), ctypes.c_uint32(b.size), _p(x))
    return None if rc != 0 else x
