"""The stage-one quasi-Newton L-BFGS-B (csrc/host/lbfgsb.cpp) on the
reference's own test problems and their expected answers
(src/numeric/lbfgsb.rs:1040-1312), including the NEBULA-shaped problem whose
values the reference pins to scipy's L-BFGS-B."""
import math

import numpy as np
import pytest

import oracle_ffi as of
from edge_rs_b200.api import NebulaError

GRADIENT, OBJECTIVE, MAX_ITER, LINE_SEARCH = 0, 1, 2, 3
INF = math.inf


def rosenbrock(x):
    a, b = x
    g = np.array([-400.0 * a * (b - a * a) - 2.0 * (1.0 - a), 200.0 * (b - a * a)])
    return 100.0 * (b - a * a) ** 2 + (1.0 - a) ** 2, g


def quadratic(x):
    d = x - np.array([1.0, 2.0, 3.0])
    return float(np.sum(d * d)), 2.0 * d


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b))


def test_unbounded_rosenbrock_finds_the_optimum():
    x, f, *_ = of.lbfgsb(rosenbrock, [-1.2, 1.0], [-INF] * 2, [INF] * 2, ftol=1e-14, pgtol=1e-10, max_iter=500)
    assert rel(x[0], 1.0) <= 1e-5 and rel(x[1], 1.0) <= 1e-5
    assert f < 1e-10


def test_quadratic_converges():
    x, *_ = of.lbfgsb(quadratic, [0.0] * 3, [-INF] * 3, [INF] * 3, ftol=1e-14, pgtol=1e-12)
    for v, want in zip(x, (1.0, 2.0, 3.0)):
        assert rel(v, want) <= 1e-8


def test_active_bound_is_respected():
    x, *_ = of.lbfgsb(quadratic, [5.0, 0.0, 0.0], [2.0, -INF, -INF], [INF] * 3, ftol=1e-14, pgtol=1e-12)
    assert rel(x[0], 2.0) <= 1e-10
    assert rel(x[1], 2.0) <= 1e-8 and rel(x[2], 3.0) <= 1e-8


def test_degenerate_box_returns_the_only_feasible_point():
    x, *_ = of.lbfgsb(quadratic, [0.0] * 3, [1.5] * 3, [1.5] * 3)
    assert all(rel(v, 1.5) <= 1e-12 for v in x)


def test_bounded_rosenbrock_stops_on_the_boundary():
    x, *_ = of.lbfgsb(rosenbrock, [-1.2, 1.0], [-INF, -INF], [0.5, INF], ftol=1e-14, pgtol=1e-10, max_iter=500)
    assert rel(x[0], 0.5) <= 1e-6
    assert rel(x[1], 0.25) <= 1e-4


def test_infeasible_start_is_clamped():
    x, *_ = of.lbfgsb(quadratic, [-50.0, 100.0, 3.0], [0.0] * 3, [10.0] * 3)
    assert np.all(x >= -1e-12) and np.all(x <= 10.0 + 1e-12)


@pytest.mark.parametrize("x0,lo,hi,code", [
    ([0.0] * 3, [1.0, 0.0, 0.0], [0.0, 1.0, 1.0], 12),  # InvalidBounds
    ([0.0] * 3, [0.0] * 2, [1.0] * 3, 2),               # LengthMismatch (lower)
    ([], [], [], 5),                                     # MustBePositive
])
def test_rejected_arguments(x0, lo, hi, code):
    with pytest.raises(NebulaError) as e:
        of.lbfgsb(quadratic, x0, lo, hi)
    assert e.value.code == code


def nebula_shaped(p):
    """The reference's NB-with-penalty problem of stage one's shape
    (lbfgsb.rs:1192-1226), parameters [beta0, beta1, sigma, phi]."""
    n = 60
    counts = [[0.0, 3.0, 1.0, 2.0, 0.0, 5.0, 2.0, 1.0, 4.0, 2.0][i % 10] for i in range(n)]
    offset = math.log(800.0)
    b0, b1, sigma, phi = p
    r = 1.0 / phi
    f = 0.5 * sigma * sigma
    gb0 = gb1 = dr = 0.0
    for i, y in enumerate(counts):
        xi = -1.0 + 2.0 * i / (n - 1)
        mu = math.exp(offset + b0 + b1 * xi)
        f += (y + r) * math.log(mu + r) - y * math.log(mu) - r * math.log(r)
        d_mu = (y + r) / (mu + r) - y / mu
        gb0 += d_mu * mu
        gb1 += xi * d_mu * mu
        dr += math.log(mu + r) + (y + r) / (mu + r) - math.log(r) - 1.0
    return f, np.array([gb0, gb1, sigma, dr * (-1.0 / (phi * phi))])


def test_nebula_shaped_problem_matches_scipy():
    # the reference's values from scipy's L-BFGS-B (lbfgsb.rs:1231-1254)
    x, f, *_ = of.lbfgsb(nebula_shaped, [0.0, 0.0, 1.0, 1.0], [-100.0, -100.0, 1e-4, 1e-4],
                         [100.0, 100.0, 10.0, 1000.0], ftol=1e-12, pgtol=1e-10, max_iter=500)
    assert rel(x[0], -5.992406750800) <= 1e-6
    assert rel(x[1], 0.074133661253) <= 1e-5
    assert rel(x[2], 1e-4) <= 1e-12
    assert rel(x[3], 1000.0) <= 1e-12
    assert rel(f, 0.516012646087) <= 1e-8


def decaying(x):
    rate = np.array([1.0, 30.0, 300.0, 3000.0])
    e = np.exp(-rate * x)
    return float(np.sum(e)), -rate * e


def test_search_stops_at_the_boundary_rather_than_past_it():
    x, f, status, iters, evals = of.lbfgsb(decaying, [0.0] * 4, [0.0] * 4, [1.0] * 4, ftol=0.0, pgtol=1e-10,
                                           max_iter=200)
    assert all(rel(v, 1.0) <= 1e-12 for v in x)
    assert status == GRADIENT
    assert evals < 100


def test_solve_dense():
    x = of.lbfgsb_solve_dense([2.0, 1.0, 1.0, 3.0], [3.0, 5.0])
    assert rel(x[0], 0.8) <= 1e-12 and rel(x[1], 1.4) <= 1e-12
    assert of.lbfgsb_solve_dense([1.0, 2.0, 2.0, 4.0], [1.0, 2.0]) is None
