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


def run(f, x0, lo, hi, radius_scale=None):
    lib = _ffi.product_library()
    n = len(x0)
    arr = lambda v: (ctypes.c_double * n)(*v)
    if radius_scale is None:
        h = lib.nb_bobyqa_new(arr(x0), arr(lo), arr(hi), n, 1e-6, 1000)
    else:
        h = lib.nb_bobyqa_new_scaled(arr(x0), arr(lo), arr(hi), n, 1e-6, 1000, radius_scale)
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


def test_scaled_radius_one_is_nlopts_search():
    for tag, f, x0, lo, hi, _ in CASES:
        a, *_ = run(f, x0, lo, hi)
        b, *_ = run(f, x0, lo, hi, radius_scale=1.0)
        assert np.array_equal(a, b), tag


def bowl(x):
    """A smooth objective shaped like the variance search's near its optimum."""
    a, b = np.log(x[0] / 0.45), np.log(x[1] / 2.0)
    return 3.0 * a * a + 0.8 * a * b + 0.5 * b * b + 0.2 * a * a * a


def test_scaled_radius_from_a_close_start_saves_evaluations():
    """From a start within 1% of the minimum, in the variance search's box,
    a search whose trust region starts at 3% of NLopt's radius ends at the
    same minimum (the final radius is NLopt's) in fewer evaluations."""
    x0, lo, hi = [0.454, 1.98], [1e-4, 1e-4], [10.0, 1000.0]
    _, x_full, f_full, n_full, _ = run(bowl, x0, lo, hi)
    _, x_warm, f_warm, n_warm, st = run(bowl, x0, lo, hi, radius_scale=0.03)
    assert st == 4  # xtol reached
    assert n_warm < 0.8 * n_full, (n_warm, n_full)
    assert np.allclose(x_warm, [0.45, 2.0], rtol=1e-5) and np.allclose(x_full, [0.45, 2.0], rtol=1e-5)
    assert f_warm < 1e-10 and f_full < 1e-10


def test_scaled_radius_still_travels_from_a_far_start():
    """A start far from the minimum with a narrow initial region: the region
    grows with successful steps and the search still reaches the minimum."""
    _, x, f, _, _ = run(rosen, [-1.2, 1.0], [-2.0, -1.0], [2.0, 3.0], radius_scale=0.03)
    assert np.allclose(x, [1.0, 1.0], atol=1e-4) and f < 1e-8
