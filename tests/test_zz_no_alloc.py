"""nb_opt_pml_cuda_noalloc (device buffers in, device buffers out, working
memory in the library's fixed scratch array) against nb_opt_pml_cuda.

Both run the same fit kernel on the same inputs, so the results must agree to
the 1e-12 relative bar the device inner-fit tests hold the profile scalars
to, with identical Newton iteration and backtrack counts. Two calls in a row
with different shapes check that nothing from the first call leaks into the
second through the shared array.
"""
import ctypes

import numpy as np
import pytest

import golden_io as gio
from device_ffi import opt_pml_batch
from edge_rs_b200 import _ffi, workloads
from pml_fixtures import centred, gene_view

REL = 1e-12
NB_ERR_INVALID_ARGUMENT = 4


def _lib():
    lib = _ffi.product_library()
    lib.nb_opt_pml_cuda_noalloc.restype = ctypes.c_int32
    return lib


def _noalloc(torch, v, n_beta, beta0, subject, cell, ords):
    """Copies one gene's inputs to the device, calls the no-allocation entry
    point and returns its outputs as host arrays in opt_pml_batch's form."""
    dev = torch.device("cuda:0")

    def put(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype)).to(dev)

    n_req = len(subject)
    design, offset = put(v["design"], np.float64), put(v["offset"], np.float64)
    counts, cells = put(v["counts"], np.float64), put(v["cells"].astype(np.int32), np.int32)
    ss, tot = put(v["subject_start"].astype(np.int64), np.int64), put(v["subject_total"], np.float64)
    b0 = put(np.broadcast_to(beta0, (n_req, n_beta)), np.float64)
    subj, cel, ordv = put(subject, np.float64), put(cell, np.float64), put(ords, np.int32)
    beta = torch.zeros(n_req * n_beta, dtype=torch.float64, device=dev)
    info = torch.zeros(n_req * n_beta * n_beta, dtype=torch.float64, device=dev)
    sc = torch.zeros(n_req * 4, dtype=torch.float64, device=dev)
    ints = torch.zeros(n_req * 4, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    err = ctypes.create_string_buffer(256)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = _lib().nb_opt_pml_cuda_noalloc(
        p(design), p(offset), ctypes.c_uint64(v["offset"].size), ctypes.c_uint32(n_beta), p(counts), p(cells),
        ctypes.c_uint64(v["counts"].size), p(ss), ctypes.c_uint32(v["subject_start"].size - 1), p(tot),
        ctypes.c_uint32(n_req), p(b0), p(subj), p(cel), p(ordv), ctypes.c_int32(0), ctypes.c_double(1e-6),
        p(beta), p(info), p(sc), p(ints), None, err, ctypes.c_size_t(len(err)))
    assert rc == 0, err.value.decode()
    beta, info, sc = beta.cpu().numpy().reshape(n_req, n_beta), info.cpu().numpy().reshape(n_req, -1), \
        sc.cpu().numpy().reshape(n_req, 4)
    ints = ints.cpu().numpy().reshape(n_req, 4)
    return [dict(beta=beta[q], information=info[q], log_likelihood=sc[q, 0], log_likelihood_prev=sc[q, 1],
                 log_det=sc[q, 2], second_order=sc[q, 3], status=int(ints[q, 0]), iterations=int(ints[q, 1]),
                 backtracks=int(ints[q, 2]), sweeps=int(ints[q, 3])) for q in range(n_req)]


def _gene(name, seed, n_cells, k, g):
    w = workloads.make(name, seed=seed, n_genes=g + 1, n_cells=n_cells, n_subjects=k)
    fid = np.concatenate([[0], np.cumsum(w.truth["sizes"])]).astype(np.uint64)
    work = dict(indptr=w.indptr, indices=w.indices, data=w.data, design_c=centred(w.design),
                log_offset=np.log(w.offset), fid=fid)
    return gene_view(work, g), w.n_coef


@pytest.mark.gpu
def test_noalloc_matches_the_allocating_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    calls = [
        (_gene("c1", 7, 12000, 12, 1), [0.2, 0.05, 1.5, 0.3, 1e-4, 9.0, 0.7, 2.5], [2.0, 0.5, 10.0, 1.0, 1000.0,
                                                                                    1e-4, 3.0, 0.2],
         [1, 1, 1, 3, 1, 2, 1, 2]),
        (_gene("c2", 3, 5000, 7, 0), [0.4, 1.1, 0.02], [5.0, 0.8, 40.0], [1, 3, 1]),
    ]
    for (v, n_beta), subject, cell, ords in calls:
        beta0 = np.zeros(n_beta)
        beta0[0] = np.log(max(v["counts"].sum() / v["offset"].size, 1e-3))
        want = opt_pml_batch(v["design"], v["offset"], n_beta, v["counts"], v["cells"], v["subject_start"],
                             v["subject_total"], beta0, subject, cell, ord=ords)
        got = _noalloc(torch, v, n_beta, beta0, subject, cell, ords)
        for q, (a, b) in enumerate(zip(got, want)):
            for key in ("status", "iterations", "backtracks", "sweeps"):
                assert a[key] == b[key], (q, key)
            for key in ("beta", "information", "log_likelihood", "log_likelihood_prev", "log_det",
                        "second_order"):
                ok, worst = gio.close(a[key], b[key], REL, 1e-12)
                assert ok, f"request {q}: {key} off by {worst:.2e}"


def test_noalloc_refuses_calls_beyond_its_scratch_before_touching_a_device():
    lib = _lib()
    err = ctypes.create_string_buffer(256)
    null = ctypes.c_void_p(0)
    rc = lib.nb_opt_pml_cuda_noalloc(null, null, ctypes.c_uint64(100), ctypes.c_uint32(2), null, null,
                                     ctypes.c_uint64(0), null, ctypes.c_uint32(4), null, ctypes.c_uint32(4096),
                                     null, null, null, null, ctypes.c_int32(0), ctypes.c_double(1e-6), null, null,
                                     null, null, None, err, ctypes.c_size_t(len(err)))
    assert rc == NB_ERR_INVALID_ARGUMENT
    assert b"at most 2048 requests" in err.value
