"""Accuracy of the shared exp/log (nbmath.hpp) that the device sweep and the
oracle both use, against 80-bit long double, plus their special values.

The bar: within 1 ulp for exp and within 2 ulp for log (the cancellation of
e ln2 against -ln inv_j just below 1 can cost one more) over the arguments
the fits see, exact at the special values.
"""
import ctypes

import numpy as np
import pytest

import oracle_ffi as of

if np.finfo(np.longdouble).nmant < 60:
    pytest.skip("needs x86 80-bit long double as the reference", allow_module_level=True)


def run(which, x):
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty_like(x)
    lib = of.lib()
    lib.oracle_nbmath(ctypes.c_int32(which), x.ctypes.data_as(ctypes.c_void_p),
                      out.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint64(x.size))
    return out


def ulp_error(got, want_ld):
    want = want_ld.astype(np.float64)
    ulp = np.spacing(np.abs(want))
    return np.abs((got.astype(np.longdouble) - want_ld) / ulp.astype(np.longdouble)).astype(np.float64)


def exp_args(rng):
    return np.concatenate([rng.uniform(-745.0, 709.7, 200000), rng.uniform(-30, 30, 200000),
                           rng.uniform(-1e-3, 1e-3, 50000), np.arange(-2000, 2000) * (np.log(2) / 256)])


def log_args(rng):
    return np.concatenate([np.exp(rng.uniform(-700, 700, 200000)), rng.uniform(0.5, 2.0, 200000),
                           1.0 + rng.uniform(-1e-6, 1e-6, 50000), rng.uniform(1e-3, 1e4, 100000),
                           np.nextafter(1.0, 0.0) - np.arange(1000) * 2.0 ** -53,
                           np.array([2.0 ** -1074, 3e-320, 2.2250738585072014e-308])])


@pytest.mark.parametrize("which", [0, 2], ids=["nb_exp", "nb_exp_tab"])
def test_exp_within_one_ulp(which):
    x = exp_args(np.random.default_rng(1))
    got = run(which, x)
    want = np.exp(x.astype(np.longdouble))
    normal = want.astype(np.float64) >= 2.2250738585072014e-308
    err = ulp_error(got[normal], want[normal])
    assert err.max() <= 1.0, err.max()
    # subnormal results: within one unit of the smallest subnormal
    sub = ~normal
    assert np.all(np.abs(got[sub] - want[sub].astype(np.float64)) <= 5e-324)


@pytest.mark.parametrize("which", [1, 3], ids=["nb_log", "nb_log_tab"])
def test_log_within_two_ulp(which):
    x = log_args(np.random.default_rng(2))
    got = run(which, x)
    want = np.log(x.astype(np.longdouble))
    err = ulp_error(got, want)
    assert err.max() <= 2.0, err.max()
    assert np.mean(err <= 0.5001) > 0.85


@pytest.mark.parametrize("which", [0, 2])
def test_exp_special_values(which):
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 710.0, -746.0, 1.0])
    got = run(which, x)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == np.inf and got[3] == 0.0
    assert np.isnan(got[4]) and got[5] == np.inf and got[6] == 0.0
    assert abs(got[7] - np.e) <= np.spacing(np.e)


@pytest.mark.parametrize("which", [1, 3])
def test_log_special_values(which):
    x = np.array([1.0, 0.0, -1.0, np.inf, np.nan, 2.0, 0.5])
    got = run(which, x)
    assert got[0] == 0.0 and got[1] == -np.inf and np.isnan(got[2]) and got[3] == np.inf
    assert np.isnan(got[4])
    assert got[5] == np.log(2.0) and got[6] == -np.log(2.0)


def test_log_table_reduction_is_exact():
    """r = m inv_j - 1 is exact: every table reciprocal has at most nine
    significant bits and |r| <= 2^-8 over each index's interval."""
    rng = np.random.default_rng(3)
    m = np.concatenate([rng.uniform(1.0, 2.0, 100000), 1.0 + (np.arange(257) - 0.5) / 256])
    m = m[(m >= 1.0) & (m < 2.0)]
    j = np.rint((m - 1.0) * 256).astype(int)
    fold = j == 256
    m = np.where(fold, m / 2, m)
    j = np.where(fold, 0, j)
    inv = np.rint(512 / (1.0 + j / 256)) / 512
    r_ld = m.astype(np.longdouble) * inv.astype(np.longdouble) - 1
    assert np.all(np.abs(r_ld) <= 2.0 ** -8)
    assert np.all(r_ld.astype(np.float64).astype(np.longdouble) == r_ld)
