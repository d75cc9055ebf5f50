"""BOBYQA retraces nloptr point for point (src/numeric/bobyqa.rs:2926-2972)."""
import ctypes
import math
import os

import numpy as np
import pytest

from edge_rs_b200 import _ffi
from golden_io import DATA


def sq(v):
    return v * v


def rosen(x):
    return 100.0 * sq(x[1] - x[0] * x[0]) + sq(1.0 - x[0])


def corner(x):
    return sq(x[0] - 3.0) + 10.0 * sq(x[1] + 1.0) + x[0] * x[1]


def ripple(x):
    u = 10000.0 * x[0] + 30000.0 * x[1]
    t = abs(u - 2.0 * math.floor((u + 1.0) / 2.0))
    return sq(x[0] - 0.25) + 2.0 * sq(x[1] + 0.125) + 0.5 * x[0] * x[1] + 0.5 * (t * t)


def valley(x):
    return sq(x[0] + x[1] - 1.0)


def chain3(x):
    return sq(x[0] - 1.0) + 100.0 * sq(x[1] - x[0] * x[0]) + sq(x[2] - x[1]) + 0.5 * sq(sq(x[2]))


# bobyqa.rs:2869-2924: objective, start, bounds, nloptr's exit status
CASES = [
    ("rosen", rosen, [-1.2, 1.0], [-2.0, -1.0], [2.0, 3.0], 4),
    ("rosen_edge", rosen, [0.4001, 0.2], [0.4, 0.2], [2.0, 2.0], 4),
    ("corner", corner, [1.0, 1.0], [0.0, 0.0], [2.0, 2.0], 4),
    ("chain3", chain3, [0.5, 2.0, -1.0], [-3.0] * 3, [3.0] * 3, 4),
    ("rescue", ripple, [-1.0, 0.25], [-2.0, -2.0], [2.0, 2.0], 4),
    ("roundoff", valley, [0.0, 0.0], [-2.0, -2.0], [2.0, 2.0], -4),
]


def run(f, x0, lo, hi):
    lib = _ffi.product_library()
    n = len(x0)
    arr = lambda v: (ctypes.c_double * n)(*v)
    h = lib.nb_bobyqa_new(arr(x0), arr(lo), arr(hi), n, 1e-6, 1000)
    assert h
    trace = []
    x = (ctypes.c_double * n)()
    while lib.nb_bobyqa_ask(h, x):
        xv = list(x)
        v = f(xv)
        trace.append(xv + [v])
        lib.nb_bobyqa_tell(h, v)
    xr = (ctypes.c_double * n)()
    fr = ctypes.c_double()
    ne = ctypes.c_uint32()
    status = lib.nb_bobyqa_result(h, xr, ctypes.byref(fr), ctypes.byref(ne))
    lib.nb_bobyqa_free(h)
    return np.array(trace), list(xr), fr.value, ne.value, status


@pytest.mark.parametrize("tag,f,x0,lo,hi,status", CASES, ids=[c[0] for c in CASES])
def test_bobyqa_retraces_nloptr_point_for_point(tag, f, x0, lo, hi, status):
    want = np.loadtxt(os.path.join(DATA, f"bobyqa_{tag}.csv"), delimiter=",", ndmin=2)
    got, _, _, nevals, st = run(f, x0, lo, hi)
    assert got.shape == want.shape
    assert np.array_equal(got, want)  # bit for bit
    assert nevals == len(want)
    assert st == status


def test_bobyqa_lands_on_an_active_bound():
    _, x, f, _, _ = run(corner, [1.0, 1.0], [0.0, 0.0], [2.0, 2.0])
    assert x == [2.0, 0.0] and f == 11.0


def test_bobyqa_refuses_a_box_narrower_than_two_radii():
    lib = _ffi.product_library()
    arr = lambda v: (ctypes.c_double * 2)(*v)
    # the initial radius is a quarter of the narrowest side; a degenerate side refuses
    assert not lib.nb_bobyqa_new(arr([0.0, 0.0]), arr([0.0, 0.0]), arr([0.0, 1.0]), 2, 1e-6, 1000)
