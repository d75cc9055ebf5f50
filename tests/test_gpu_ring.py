"""The request ring that feeds the persistent kernels, on the device
(nb_ring_check_cuda: the same host queue and device protocol, served by an
echo kernel). Every ticket is answered once and correctly, also when the
ring has far fewer slots than requests; and a wait for work that runs out
ends the kernel with an error status the host reports as NB_ERR_GPU, with no
device fault, after which the device serves the next call normally."""
import ctypes
import time

import pytest

from edge_rs_b200 import _ffi

pytestmark = pytest.mark.gpu


def ring_check(n_requests, capacity, ctas, idle_ms=0):
    lib = _ffi.product_library()
    bad = ctypes.c_uint64(123)
    err = ctypes.create_string_buffer(512)
    rc = lib.nb_ring_check_cuda(n_requests, capacity, ctas, idle_ms, ctypes.byref(bad), err, len(err))
    return _ffi.STATUS_NAMES[rc], bad.value, err.value.decode()


@pytest.mark.parametrize("n_requests, capacity, ctas", [
    (1, 2, 1),
    (100_000, 16384, 296),    # the fit queue's ring size
    (200_000, 256, 296),      # more waiting CTAs than slots: every slot reused ~800 times
    (50_000, 64, 4),
])
def test_every_ticket_is_answered_once_and_correctly(n_requests, capacity, ctas):
    status, bad, err = ring_check(n_requests, capacity, ctas)
    assert status == "Ok", err
    assert bad == 0


def test_a_wait_for_work_that_runs_out_is_an_error_not_a_fault():
    t0 = time.perf_counter()
    status, _, err = ring_check(0, 1024, 148, idle_ms=200)
    elapsed = time.perf_counter() - t0
    assert status == "Gpu", err
    assert "waited more than 200 ms for work" in err
    assert elapsed < 10.0
    # the context is intact: the next call runs normally
    status, bad, err = ring_check(20_000, 1024, 148)
    assert status == "Ok" and bad == 0, err


def test_bad_arguments_are_refused_before_any_launch():
    assert ring_check(10, 1000, 4)[0] == "InvalidArgument"  # not a power of two
    assert ring_check(10, 1024, 0)[0] == "InvalidArgument"
