"""Python mirror of edge-rs's NEBULA interface for the B200 path.

`nebula_sparse_cuda` takes what `nebula_sparse` takes (src/sc/nebula.rs:434-445:
gene-major CSR counts, contiguous subject ids, a design with an intercept of
up to 8 columns, optional positive offsets, NebulaParams) and returns the same
NebulaFit (nebula.rs:301-344). It calls the C-ABI of libnebula_b200.so; there
is no CPU fallback. Errors raise NebulaError carrying the EdgeErrors variant.
"""
import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _ffi


class NebulaError(RuntimeError):
    """An EdgeErrors value returned through the C-ABI."""

    def __init__(self, code, message):
        self.code = int(code)
        self.variant = _ffi.STATUS_NAMES.get(self.code, f"code {code}")
        super().__init__(f"{self.variant}: {message}")


@dataclass
class NebulaParams:
    """NebulaParams (nebula.rs:207-258); defaults are the R package's."""
    min: tuple = (1e-4, 1e-4)
    max: tuple = (10.0, 1000.0)
    method: str = "LN"
    cutoff_cell: float = 20.0
    kappa: float = 800.0
    cpc: float = 0.005
    mincp: int = 5
    min_subjects: int = 0
    reml: bool = False
    eps: float = 1e-6

    def to_c(self):
        method = {"LN": _ffi.NB_METHOD_LN, "HL": _ffi.NB_METHOD_HL}[self.method.upper()]
        return _ffi.NbParams(float(self.min[0]), float(self.min[1]), float(self.max[0]),
                             float(self.max[1]), method, float(self.cutoff_cell), float(self.kappa),
                             float(self.cpc), int(self.mincp), int(self.min_subjects),
                             int(bool(self.reml)), float(self.eps))


@dataclass
class NebulaFit:
    """NebulaFit (nebula.rs:301-344); covariance packed upper column-major."""
    coefficients: np.ndarray
    covariance: np.ndarray
    se: np.ndarray
    subject_overdispersion: np.ndarray
    cell_overdispersion: np.ndarray
    convergence: np.ndarray
    sigma_at_bound: np.ndarray
    gene_index: np.ndarray
    n_coef: int
    stats: dict = field(default_factory=dict)
    evaluations: Optional[np.ndarray] = None  # stage-two objective evaluations per gene


def _as_csr(counts):
    """(indptr, indices, data, shape) from a scipy CSR matrix or a 4-tuple."""
    if hasattr(counts, "indptr") and hasattr(counts, "indices"):
        fmt = _ffi.NB_CSR if getattr(counts, "format", "csr") == "csr" else _ffi.NB_CSC
        return _ffi.CsrArrays(counts.indptr, counts.indices, counts.data, counts.shape, fmt)
    indptr, indices, data, shape = counts
    return _ffi.CsrArrays(indptr, indices, data, shape)


def fit_from_arrays(f, n_coef, stats=None):
    n = int(f.struct.n_kept)
    packed = n_coef * (n_coef + 1) // 2
    return NebulaFit(
        coefficients=f.coefficients[: n * n_coef].reshape(n, n_coef).copy(),
        covariance=f.covariance[: n * packed].reshape(n, packed).copy(),
        se=f.se[: n * n_coef].reshape(n, n_coef).copy(),
        subject_overdispersion=f.subject[:n].copy(),
        cell_overdispersion=f.cell[:n].copy(),
        convergence=f.convergence[:n].copy(),
        sigma_at_bound=f.at_bound[:n].astype(bool),
        gene_index=f.gene_index[:n].astype(np.int64),
        n_coef=int(f.struct.n_coef),
        stats=stats or {},
    )


def call_nebula(fn, counts, subject_id, design, n_coef, offset, params, extra_args=(), options=None,
                want_stats=False):
    """Marshals the arguments of a nebula_sparse-shaped C entry point."""
    csr = _as_csr(counts)
    n_genes, n_cells = int(csr.struct.n_genes), int(csr.struct.n_cells)
    subject = np.ascontiguousarray(subject_id, dtype=np.uint64)
    design = np.ascontiguousarray(design, dtype=np.float64).reshape(-1)
    off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float64)
    if subject.size != n_cells:
        raise NebulaError(2, f"subject_id has {subject.size} entries, expected {n_cells}")
    if design.size != n_cells * n_coef:
        raise NebulaError(3, f"design has {design.size} values, expected {n_cells * n_coef}")
    if off is not None and off.size != n_cells:
        raise NebulaError(2, f"offset has {off.size} entries, expected {n_cells}")
    p = (params or NebulaParams()).to_c()
    out = _ffi.FitArrays(n_genes, n_coef)
    err = ctypes.create_string_buffer(512)
    stats = _ffi.NbStats()
    args = [ctypes.byref(csr.struct), _ffi.ptr(subject, ctypes.c_uint64), _ffi.ptr(design, ctypes.c_double),
            ctypes.c_uint32(n_coef), _ffi.ptr(off, ctypes.c_double), ctypes.byref(p)]
    if options is not None:
        args.append(ctypes.byref(options))
    args += list(extra_args)
    args.append(ctypes.byref(out.struct))
    if want_stats:
        args.append(ctypes.byref(stats))
    args += [err, ctypes.c_size_t(len(err))]
    rc = fn(*args)
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return fit_from_arrays(out, n_coef, stats.as_dict() if want_stats else None)


def _options(device, warm_start, host_threads, audit_percent, cluster, n_genes, warm_points=None,
             mlp_weights=None, warm_radius=0.0, dense_sweep=False, cold_inner=False):
    """An NbOptions plus the arrays it points into (kept alive by the caller)."""
    evaluations = np.zeros(max(int(n_genes), 1), np.int32)
    wp = None if warm_points is None else np.ascontiguousarray(warm_points, np.float64).reshape(-1, 2)
    mw = None if mlp_weights is None else np.ascontiguousarray(mlp_weights, np.float32)
    if mw is not None and mw.size != _ffi.MLP_PARAMS:
        raise NebulaError(2, f"mlp_weights has {mw.size} values, expected {_ffi.MLP_PARAMS}")
    if wp is not None and wp.shape[0] != n_genes:
        raise NebulaError(2, f"warm_points has {wp.shape[0]} rows, expected {n_genes}")
    mode = int(warm_start)
    opts = _ffi.NbOptions(int(device), mode, int(host_threads), int(audit_percent),
                          _ffi.ptr(mw, ctypes.c_float), int(cluster), _ffi.ptr(wp, ctypes.c_double),
                          _ffi.ptr(evaluations, ctypes.c_int32), float(warm_radius), int(bool(dense_sweep)),
                          int(bool(cold_inner)))
    return opts, [evaluations, wp, mw]


def nebula_sparse_cuda(counts, subject_id, design, n_coef, offset=None, params: Optional[NebulaParams] = None,
                       warm_start=False, device=-1, host_threads=0, audit_percent=5, cluster=0, warm_points=None,
                       mlp_weights=None, warm_radius=0.0, dense_sweep=False, cold_inner=False):
    """Fits NEBULA per gene with every inner penalised fit on the GPU.

    warm_start: False/0 plain (the reference's method). Otherwise every
    inner fit after a gene's first search step starts from the gene's
    previous iterate, and the search starts from: True/1 the warm-start
    network's prediction (`mlp_weights`, or the built-in network); 2
    `warm_points` (n_genes x (sigma, gamma)); 3 stage one's estimate.
    audit_percent of the searched genes also run plain and keep that
    result when its objective is better. warm_radius: the warm search's
    initial BOBYQA trust radius as a fraction of NLopt's (0: the library's
    default; 1: NLopt's); the final radius is NLopt's either way.
    dense_sweep: visit every cell in every sweep even where the zero-count
    tables of a categorical design apply (by default they are used, as the
    reference's CPU path uses them). cold_inner: with a warm start, every
    inner fit still starts cold, as the plain method's do (with
    warm_radius=1 and audit_percent=0 the search then differs from the
    plain one only in where it starts).
    """
    lib = _ffi.product_library()
    n_genes = int(_as_csr(counts).struct.n_genes)
    opts, keep = _options(device, warm_start, host_threads, audit_percent, cluster, n_genes, warm_points,
                          mlp_weights, warm_radius, dense_sweep, cold_inner)
    fit = call_nebula(lib.nebula_sparse_cuda_ex, counts, subject_id, design, n_coef, offset, params,
                      options=opts, want_stats=True)
    fit.evaluations = keep[0][: len(fit.gene_index)].copy()
    return fit


@dataclass
class ScTestResult:
    """glm_sc_test's output (src/sc/test.rs:69-82) plus log p-values."""
    log_fc: np.ndarray
    se: np.ndarray
    z: np.ndarray
    p_value: np.ndarray
    log_p_value: np.ndarray
    fdr: np.ndarray


def glm_sc_test(coefficients, covariance, coef=None, contrast=None):
    """Wald test of one coefficient or a contrast per gene (src/sc/test.rs:96-200)."""
    lib = _ffi.product_library()
    beta = np.ascontiguousarray(coefficients, dtype=np.float64)
    n_genes, n_coef = beta.shape
    cov = np.ascontiguousarray(covariance, dtype=np.float64)
    if contrast is None:
        if coef is None or not 0 <= coef < n_coef:
            raise NebulaError(13, f"coefficient {coef} is out of range for {n_coef}")
        contrast = np.zeros(n_coef)
        contrast[coef] = 1.0
    c = np.ascontiguousarray(contrast, dtype=np.float64)
    outs = [np.zeros(n_genes) for _ in range(6)]
    err = ctypes.create_string_buffer(256)
    rc = lib.nb_glm_sc_test(_ffi.ptr(beta, ctypes.c_double), _ffi.ptr(cov, ctypes.c_double), n_genes, n_coef,
                            _ffi.ptr(c, ctypes.c_double), *[_ffi.ptr(o, ctypes.c_double) for o in outs],
                            err, len(err))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return ScTestResult(*outs)


def glm_sc_test_cuda(coefficients, covariance, coef=None, contrast=None):
    """glm_sc_test on the device for fits held in HBM: `coefficients`
    (n_genes x n_coef) and the packed `covariance` are CUDA float64 tensors;
    returns an ScTestResult of CUDA tensors (nb_glm_sc_test_cuda)."""
    import torch
    lib = _ffi.product_library()
    beta = coefficients.contiguous()
    cov = covariance.contiguous()
    if not (beta.is_cuda and cov.is_cuda) or beta.dtype != torch.float64 or cov.dtype != torch.float64:
        raise NebulaError(2, "coefficients and covariance must be CUDA float64 tensors")
    n_genes, n_coef = beta.shape
    if contrast is None:
        if coef is None or not 0 <= coef < n_coef:
            raise NebulaError(13, f"coefficient {coef} is out of range for {n_coef}")
        contrast = np.zeros(n_coef)
        contrast[coef] = 1.0
    c = np.ascontiguousarray(contrast, dtype=np.float64)
    outs = [torch.empty(n_genes, dtype=torch.float64, device=beta.device) for _ in range(6)]
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream(beta.device).cuda_stream
    rc = lib.nb_glm_sc_test_cuda(beta.data_ptr(), cov.data_ptr(), n_genes, n_coef, _ffi.ptr(c, ctypes.c_double),
                                 *[o.data_ptr() for o in outs], ctypes.c_void_p(stream), err, len(err))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return ScTestResult(*outs)


CONTRACT_VARIANTS = {0: "fp64_cuda_cores", 1: "fp32_cuda_cores", 2: "tf32_tensor_cores", 3: "split_bf16_tensor_cores"}


def contract_krx_cuda(variant, design, weights):
    """S[r] = sum_c weights[r, c] x_c x_c' packed (b (b + 1) / 2 + a for
    a <= b) for CUDA float64 tensors design (n_cells x p, p <= 8) and
    weights (R x n_cells, R <= 128), in one of CONTRACT_VARIANTS
    (nb_contract_krx_cuda). Returns (S as a CUDA tensor, contraction ms,
    ms with the operand conversions)."""
    import torch
    lib = _ffi.product_library()
    x = design.contiguous()
    w = weights.contiguous()
    if not (x.is_cuda and w.is_cuda) or x.dtype != torch.float64 or w.dtype != torch.float64:
        raise NebulaError(2, "design and weights must be CUDA float64 tensors")
    n_cells, p = x.shape
    r = w.shape[0]
    out = torch.empty((r, p * (p + 1) // 2), dtype=torch.float64, device=x.device)
    ms = np.zeros(2)
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    rc = lib.nb_contract_krx_cuda(int(variant), x.data_ptr(), n_cells, p, w.data_ptr(), r, out.data_ptr(),
                                  _ffi.ptr(ms, ctypes.c_double), ctypes.c_void_p(stream), err, len(err))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return out, float(ms[0]), float(ms[1])


class Session:
    """nb_session_create / nb_session_fit: inputs validated, stage one run and
    the data made resident on the device once; `fit()` runs stages two and
    three on the resident copy."""

    def __init__(self, counts, subject_id, design, n_coef, offset=None, params: Optional[NebulaParams] = None,
                 warm_start=False, device=-1, host_threads=0, audit_percent=5, cluster=0, warm_points=None,
                 mlp_weights=None, warm_radius=0.0, dense_sweep=False, cold_inner=False):
        self._lib = _ffi.product_library()
        self._keep = []
        csr = _as_csr(counts)
        subject = np.ascontiguousarray(subject_id, dtype=np.uint64)
        design = np.ascontiguousarray(design, dtype=np.float64).reshape(-1)
        off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float64)
        self.n_genes = int(csr.struct.n_genes)
        self.n_coef = int(n_coef)
        p = (params or NebulaParams()).to_c()
        opts, arrays = _options(device, warm_start, host_threads, audit_percent, cluster, self.n_genes,
                                warm_points, mlp_weights, warm_radius, dense_sweep, cold_inner)
        self._evaluations = arrays[0]
        self._keep = [csr, subject, design, off, p, opts, arrays]
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._lib.nb_session_create(ctypes.byref(csr.struct), _ffi.ptr(subject, ctypes.c_uint64),
                                         _ffi.ptr(design, ctypes.c_double), ctypes.c_uint32(n_coef),
                                         _ffi.ptr(off, ctypes.c_double), ctypes.byref(p), ctypes.byref(opts),
                                         ctypes.byref(handle), err, len(err))
        if rc != 0:
            raise NebulaError(rc, err.value.decode(errors="replace"))
        self._handle = handle

    def fit(self):
        out = _ffi.FitArrays(self.n_genes, self.n_coef)
        stats = _ffi.NbStats()
        err = ctypes.create_string_buffer(512)
        rc = self._lib.nb_session_fit(self._handle, ctypes.byref(out.struct), ctypes.byref(stats), err, len(err))
        if rc != 0:
            raise NebulaError(rc, err.value.decode(errors="replace"))
        fit = fit_from_arrays(out, self.n_coef, stats.as_dict())
        fit.evaluations = self._evaluations[: len(fit.gene_index)].copy()
        return fit

    def features(self):
        """The kept genes' warm-start features (n_kept x 12) and stage one's
        (sigma, gamma) (n_kept x 2)."""
        n = ctypes.c_uint64(0)
        err = ctypes.create_string_buffer(256)
        feats = np.zeros((self.n_genes, _ffi.MLP_FEATURES), np.float32)
        s1 = np.zeros((self.n_genes, 2))
        rc = self._lib.nb_session_features(self._handle, _ffi.ptr(feats, ctypes.c_float), _ffi.ptr(s1, ctypes.c_double),
                                           ctypes.byref(n), err, len(err))
        if rc != 0:
            raise NebulaError(rc, err.value.decode(errors="replace"))
        return feats[: n.value].copy(), s1[: n.value].copy()

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.nb_session_free(self._handle)
            self._handle = None

    def __del__(self):
        self.close()


def opt_pml_cuda(design, offset, counts, cells, subject_start, subject_total, beta_init, subject, cell, ord=None,
                 reml=False, eps=1e-6):
    """A batch of inner fits of one gene on the GPU (nb_opt_pml_cuda; the
    reference's opt_pml, src/sc/pml.rs:468-508, once per (subject, cell)
    point). `design` is used as given (n_cells x n_beta), `offset` holds log
    offsets, `counts`/`cells` the positive entries in cell order,
    `subject_start` the k + 1 subject boundaries. Returns a dict of arrays:
    beta (n x n_beta), information (n x n_beta^2), log_likelihood,
    log_likelihood_prev, log_det, second_order, status, iterations,
    backtracks, sweeps."""
    lib = _ffi.product_library()
    design = np.ascontiguousarray(design, np.float64)
    offset = np.ascontiguousarray(offset, np.float64)
    n_cells = offset.size
    n_beta = design.size // n_cells
    counts = np.ascontiguousarray(counts, np.float64)
    cells = np.ascontiguousarray(cells, np.uint32)
    ss = np.ascontiguousarray(subject_start, np.uint64)
    tot = np.ascontiguousarray(subject_total, np.float64)
    subject = np.atleast_1d(np.asarray(subject, np.float64))
    n = subject.size
    cell = np.ascontiguousarray(np.broadcast_to(np.asarray(cell, np.float64), (n,)))
    b0 = np.ascontiguousarray(np.broadcast_to(np.asarray(beta_init, np.float64), (n, n_beta)))
    ordv = np.ascontiguousarray(np.broadcast_to(np.asarray(1 if ord is None else ord, np.int32), (n,)))
    beta = np.zeros((n, n_beta))
    info = np.zeros((n, n_beta * n_beta))
    sc = np.zeros((n, 4))
    ints = np.zeros((n, 4), np.int32)
    err = ctypes.create_string_buffer(256)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.nb_opt_pml_cuda(p(design), p(offset), ctypes.c_uint64(n_cells), ctypes.c_uint32(n_beta), p(counts),
                             p(cells), ctypes.c_uint64(counts.size), p(ss), ctypes.c_uint32(ss.size - 1), p(tot),
                             ctypes.c_uint32(n), p(b0), p(subject), p(cell), p(ordv), ctypes.c_int32(int(reml)),
                             ctypes.c_double(eps), p(beta), p(info), p(sc), p(ints), err, ctypes.c_size_t(len(err)))
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))
    return dict(beta=beta, information=info, log_likelihood=sc[:, 0], log_likelihood_prev=sc[:, 1],
                log_det=sc[:, 2], second_order=sc[:, 3], status=ints[:, 0], iterations=ints[:, 1],
                backtracks=ints[:, 2], sweeps=ints[:, 3])


def _check(rc, err):
    if rc != 0:
        raise NebulaError(rc, err.value.decode(errors="replace"))


def mlp_init(seed=0):
    """Initial warm-start network parameters (NB_MLP_PARAMS float32)."""
    p = np.zeros(_ffi.MLP_PARAMS, np.float32)
    _ffi.product_library().nb_mlp_init(ctypes.c_uint64(seed), _ffi.ptr(p, ctypes.c_float))
    return p


def mlp_builtin():
    """The built-in warm-start network's parameters."""
    p = np.zeros(_ffi.MLP_PARAMS, np.float32)
    _ffi.product_library().nb_mlp_builtin(_ffi.ptr(p, ctypes.c_float))
    return p


def mlp_predict(params, features):
    """The network's outputs (n x 3) on the GPU."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, _ffi.MLP_FEATURES)
    out = np.zeros((x.shape[0], _ffi.MLP_OUTPUTS), np.float32)
    err = ctypes.create_string_buffer(256)
    _check(_ffi.product_library().nb_mlp_predict_cuda(_ffi.ptr(p, ctypes.c_float), _ffi.ptr(x, ctypes.c_float),
                                                      x.shape[0], _ffi.ptr(out, ctypes.c_float), err, len(err)), err)
    return out


def mlp_gradient(params, features, targets):
    """(loss, gradient) of the network on the GPU."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, _ffi.MLP_FEATURES)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1, _ffi.MLP_OUTPUTS)
    g = np.zeros(_ffi.MLP_PARAMS, np.float32)
    loss = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(256)
    _check(_ffi.product_library().nb_mlp_gradient_cuda(_ffi.ptr(p, ctypes.c_float), _ffi.ptr(x, ctypes.c_float),
                                                       _ffi.ptr(t, ctypes.c_float), x.shape[0],
                                                       _ffi.ptr(g, ctypes.c_float), ctypes.byref(loss), err,
                                                       len(err)), err)
    return loss.value, g


def mlp_train(features, targets, params, epochs=200, batch=512, lr=1e-3, seed=0):
    """Trains a copy of `params` with Adam on the GPU; returns (params, per-epoch mean batch loss)."""
    p = np.array(params, np.float32, copy=True)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, _ffi.MLP_FEATURES)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1, _ffi.MLP_OUTPUTS)
    losses = np.zeros(int(epochs))
    err = ctypes.create_string_buffer(256)
    _check(_ffi.product_library().nb_mlp_train_cuda(_ffi.ptr(x, ctypes.c_float), _ffi.ptr(t, ctypes.c_float),
                                                    x.shape[0], int(epochs), int(batch), ctypes.c_float(lr),
                                                    ctypes.c_uint64(seed), _ffi.ptr(p, ctypes.c_float),
                                                    _ffi.ptr(losses, ctypes.c_double), err, len(err)), err)
    return p, losses


def measure_fp64_tflops(repeats=5):
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    return float(_ffi.product_library().nb_measure_fp64_tflops(int(repeats)))
