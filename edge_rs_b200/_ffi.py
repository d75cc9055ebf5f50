"""ctypes bindings for the C-ABI in include/nebula_cuda.h.

The structs mirror the header field for field. `load_library` opens a built
shared object and declares the signatures of the entry points it exports.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(HERE, "lib", "libnebula_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_u64_p = ctypes.POINTER(ctypes.c_uint64)
c_i32_p = ctypes.POINTER(ctypes.c_int32)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)
c_float_p = ctypes.POINTER(ctypes.c_float)

NB_CSR, NB_CSC = 0, 1
NB_METHOD_LN, NB_METHOD_HL = 0, 1

STATUS_NAMES = {
    0: "Ok", 1: "EmptyCounts", 2: "LengthMismatch", 3: "ShapeMismatch", 4: "InvalidArgument",
    5: "MustBePositive", 6: "MalformedSparse", 7: "NoGenesAfterFiltering", 8: "InvalidDispersion",
    9: "SubjectsNotContiguous", 10: "MissingIntercept", 11: "TooFewSubjects", 12: "InvalidBounds",
    13: "CoefOutOfRange", 14: "Gpu", 15: "Unsupported",
}


class NbCsr(ctypes.Structure):
    _fields_ = [("n_genes", ctypes.c_uint64), ("n_cells", ctypes.c_uint64), ("nnz", ctypes.c_uint64),
                ("indptr", c_u32_p), ("indices", c_u32_p), ("data", c_double_p),
                ("format", ctypes.c_int32)]


class NbParams(ctypes.Structure):
    _fields_ = [("min_subject", ctypes.c_double), ("min_cell", ctypes.c_double),
                ("max_subject", ctypes.c_double), ("max_cell", ctypes.c_double),
                ("method", ctypes.c_int32), ("cutoff_cell", ctypes.c_double),
                ("kappa", ctypes.c_double), ("cpc", ctypes.c_double),
                ("mincp", ctypes.c_uint64), ("min_subjects", ctypes.c_uint64),
                ("reml", ctypes.c_int32), ("eps", ctypes.c_double)]


class NbFit(ctypes.Structure):
    _fields_ = [("coefficients", c_double_p), ("covariance", c_double_p), ("se", c_double_p),
                ("subject_overdispersion", c_double_p), ("cell_overdispersion", c_double_p),
                ("convergence", c_i32_p), ("sigma_at_bound", c_u8_p), ("gene_index", c_u64_p),
                ("n_kept", ctypes.c_uint64), ("n_coef", ctypes.c_uint64)]


class NbOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("warm_start", ctypes.c_int32),
                ("host_threads", ctypes.c_int32), ("audit_percent", ctypes.c_int32),
                ("mlp_weights", c_float_p), ("cluster", ctypes.c_int32),
                ("warm_points", ctypes.POINTER(ctypes.c_double)), ("evaluations", ctypes.POINTER(ctypes.c_int32)),
                ("warm_radius", ctypes.c_double), ("dense_sweep", ctypes.c_int32),
                ("cold_inner", ctypes.c_int32)]


class NbStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_uint64), ("requests", ctypes.c_uint64),
                ("sweeps", ctypes.c_uint64), ("cell_visits", ctypes.c_uint64),
                ("gpu_launches", ctypes.c_uint64), ("ms_total", ctypes.c_double),
                ("ms_prepare", ctypes.c_double), ("ms_stage_one", ctypes.c_double),
                ("ms_stage_two", ctypes.c_double), ("ms_stage_three", ctypes.c_double),
                ("ms_device", ctypes.c_double), ("ms_step_device", ctypes.c_double),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("audited", ctypes.c_uint64), ("refit_cold", ctypes.c_uint64),
                ("fit_slots", ctypes.c_uint64), ("slot_cycles", ctypes.c_uint64),
                ("cluster", ctypes.c_uint64), ("ms_upload", ctypes.c_double),
                ("ms_busy_span", ctypes.c_double), ("zero_groups", ctypes.c_uint64),
                ("ms_ticket_wait", ctypes.c_double), ("sparse_visits", ctypes.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every C-ABI entry point of the product library with its signature; the
# CPU tests check the built library exports each of them.
PRODUCT_SIGNATURES = {
    "nb_params_default": (None, [ctypes.POINTER(NbParams)]),
    "nebula_sparse_cuda": (ctypes.c_int32, [ctypes.POINTER(NbCsr), c_u64_p, c_double_p,
                                            ctypes.c_uint32, c_double_p, ctypes.POINTER(NbParams),
                                            ctypes.POINTER(NbFit), ctypes.c_char_p, ctypes.c_size_t]),
    "nebula_sparse_cuda_ex": (ctypes.c_int32, [ctypes.POINTER(NbCsr), c_u64_p, c_double_p,
                                               ctypes.c_uint32, c_double_p,
                                               ctypes.POINTER(NbParams), ctypes.POINTER(NbOptions),
                                               ctypes.POINTER(NbFit), ctypes.POINTER(NbStats),
                                               ctypes.c_char_p, ctypes.c_size_t]),
    "nb_session_create": (ctypes.c_int32, [ctypes.POINTER(NbCsr), c_u64_p, c_double_p, ctypes.c_uint32,
                                           c_double_p, ctypes.POINTER(NbParams), ctypes.POINTER(NbOptions),
                                           ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]),
    "nb_session_fit": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(NbFit), ctypes.POINTER(NbStats),
                                        ctypes.c_char_p, ctypes.c_size_t]),
    "nb_session_free": (None, [ctypes.c_void_p]),
    "nb_glm_sc_test": (ctypes.c_int32, [c_double_p, c_double_p, ctypes.c_uint64, ctypes.c_uint64,
                                        c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                                        c_double_p, c_double_p, ctypes.c_char_p, ctypes.c_size_t]),
    "nb_glm_sc_test_cuda": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                             c_double_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_char_p, ctypes.c_size_t]),
    "nb_contract_krx_cuda": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                              ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, c_double_p,
                                              ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "nb_bobyqa_new": (ctypes.c_void_p, [c_double_p, c_double_p, c_double_p, ctypes.c_uint32,
                                        ctypes.c_double, ctypes.c_uint32]),
    "nb_bobyqa_new_scaled": (ctypes.c_void_p, [c_double_p, c_double_p, c_double_p, ctypes.c_uint32,
                                               ctypes.c_double, ctypes.c_uint32, ctypes.c_double]),
    "nb_bobyqa_ask": (ctypes.c_int32, [ctypes.c_void_p, c_double_p]),
    "nb_bobyqa_tell": (None, [ctypes.c_void_p, ctypes.c_double]),
    "nb_bobyqa_result": (ctypes.c_int32, [ctypes.c_void_p, c_double_p, c_double_p,
                                          ctypes.POINTER(ctypes.c_uint32)]),
    "nb_bobyqa_free": (None, [ctypes.c_void_p]),
    "nb_search_new": (ctypes.c_void_p, [c_double_p, c_double_p, c_double_p, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_double]),
    "nb_search_ask": (ctypes.c_uint32, [ctypes.c_void_p, c_double_p, ctypes.c_uint32]),
    "nb_search_tell": (ctypes.c_int32, [ctypes.c_void_p, c_double_p, ctypes.c_uint32]),
    "nb_search_order": (ctypes.c_uint32, [ctypes.c_void_p]),
    "nb_search_result": (ctypes.c_int32, [ctypes.c_void_p, c_double_p, ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_uint32)]),
    "nb_search_free": (None, [ctypes.c_void_p]),
    "nb_ring_check_cuda": (ctypes.c_int32, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_size_t]),
    "nb_measure_fp64_tflops":(ctypes.c_double, [ctypes.c_int]),
    "nb_mlp_init": (None, [ctypes.c_uint64, c_float_p]),
    "nb_mlp_builtin": (None, [c_float_p]),
    "nb_mlp_predict_cuda": (ctypes.c_int32, [c_float_p, c_float_p, ctypes.c_uint64, c_float_p, ctypes.c_char_p,
                                             ctypes.c_size_t]),
    "nb_mlp_gradient_cuda": (ctypes.c_int32, [c_float_p, c_float_p, c_float_p, ctypes.c_uint64, c_float_p,
                                              c_double_p, ctypes.c_char_p, ctypes.c_size_t]),
    "nb_mlp_train_cuda": (ctypes.c_int32, [c_float_p, c_float_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_float, ctypes.c_uint64, c_float_p, c_double_p, ctypes.c_char_p,
                                           ctypes.c_size_t]),
    "nb_session_features": (ctypes.c_int32, [ctypes.c_void_p, c_float_p, c_double_p, c_u64_p, ctypes.c_char_p,
                                             ctypes.c_size_t]),
}

MLP_FEATURES = 12
MLP_OUTPUTS = 3
MLP_PARAMS = 5211


def declare(lib, signatures):
    for name, (restype, argtypes) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


_PRODUCT = None


def product_library():
    """The product library; raises if it has not been built (no fallback)."""
    global _PRODUCT
    if _PRODUCT is None:
        if not os.path.exists(PRODUCT_LIB):
            raise RuntimeError(f"{PRODUCT_LIB} is missing: build it with `make -C edge_rs_b200/csrc`")
        _PRODUCT = declare(ctypes.CDLL(PRODUCT_LIB), PRODUCT_SIGNATURES)
    return _PRODUCT


def ptr(array, ctype):
    if array is None:
        return None
    return array.ctypes.data_as(ctypes.POINTER(ctype))


class CsrArrays:
    """Keeps the contiguous arrays an NbCsr points into alive."""

    def __init__(self, indptr, indices, data, shape, fmt=NB_CSR):
        self.indptr = np.ascontiguousarray(indptr, dtype=np.uint32)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(data, dtype=np.float64)
        self.struct = NbCsr(int(shape[0]), int(shape[1]), int(self.data.size),
                            ptr(self.indptr, ctypes.c_uint32), ptr(self.indices, ctypes.c_uint32),
                            ptr(self.data, ctypes.c_double), int(fmt))


class FitArrays:
    """Caller-allocated NebulaFit buffers for n_genes rows."""

    def __init__(self, n_genes, n_coef):
        packed = n_coef * (n_coef + 1) // 2
        self.coefficients = np.zeros(n_genes * n_coef)
        self.covariance = np.zeros(n_genes * packed)
        self.se = np.zeros(n_genes * n_coef)
        self.subject = np.zeros(n_genes)
        self.cell = np.zeros(n_genes)
        self.convergence = np.zeros(n_genes, dtype=np.int32)
        self.at_bound = np.zeros(n_genes, dtype=np.uint8)
        self.gene_index = np.zeros(n_genes, dtype=np.uint64)
        self.struct = NbFit(ptr(self.coefficients, ctypes.c_double), ptr(self.covariance, ctypes.c_double),
                            ptr(self.se, ctypes.c_double), ptr(self.subject, ctypes.c_double),
                            ptr(self.cell, ctypes.c_double), ptr(self.convergence, ctypes.c_int32),
                            ptr(self.at_bound, ctypes.c_uint8), ptr(self.gene_index, ctypes.c_uint64),
                            0, 0)
