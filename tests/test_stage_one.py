"""Stage one's marginal likelihood against nebula's ptmg goldens (src/sc/ptmg.rs:2142-2442).

Reference values are nebula:::ptmg_ll_der_hes_eigen with R/ptmg.R's
gamma-function corrections, at 1e-10 on value and gradient and 1e-8 on the
Hessian (1e-8 / 1e-6 at the lower bound on sigma), the reference's own gates.
"""
import ctypes

import numpy as np
import pytest

import golden_io as gio
import oracle_ffi as of

CASES = gio.inline()["ptmg_cases"]


def fixture(name):
    f = gio.inline()["ptmg_fixtures"][name]
    x = np.array(f["x"], dtype=np.float64)
    design = np.column_stack([np.ones(x.shape[0]), x])
    return (np.ascontiguousarray(design), np.array(f["log_offset"]), np.array(f["counts"]),
            np.array(f["cells"], np.uint32), np.array(f["subject_totals"]), np.array(f["fid"], np.uint64))


def evaluate(name, params):
    design, log_offset, counts, cells, totals, fid = fixture(name)
    nb = design.shape[1]
    p = np.ascontiguousarray(params, np.float64)
    grad = np.zeros(nb + 2)
    hess = np.zeros((nb + 2) ** 2)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib = of.lib()
    lib.oracle_ptmg_eval.restype = ctypes.c_double
    value = lib.oracle_ptmg_eval(vp(design), vp(log_offset), ctypes.c_uint64(log_offset.size), ctypes.c_uint32(nb),
                                 vp(counts), vp(cells), ctypes.c_uint64(counts.size), vp(fid),
                                 ctypes.c_uint32(fid.size - 1), vp(totals), vp(p), vp(grad), vp(hess))
    return value, grad, hess


@pytest.mark.parametrize("case", CASES, ids=[c["src"].split(":")[-1] for c in CASES])
def test_marginal_likelihood_matches_nebula(case):
    value, grad, hess = evaluate(case["fixture"], case["params"])
    assert gio.close(value, case["value"], 1e-10 if case["gtol"] == 1e-10 else 1e-8)[0]
    ok, worst = gio.close(grad, case["gradient"], case["gtol"], 1e-12)
    assert ok, f"gradient off by {worst:.2e}"
    ok, worst = gio.close(hess, case["hessian"], case["htol"], 1e-12)
    assert ok, f"Hessian off by {worst:.2e}"
    h = hess.reshape(len(grad), len(grad))
    assert np.array_equal(h, h.T)


def test_gradient_agrees_with_finite_differences():
    params = np.array([0.25, -0.5, 0.75, 1.5, 3.0])
    _, grad, hess = evaluate("B", params)
    h = 1e-6
    for j in range(params.size):
        e = np.zeros_like(params)
        e[j] = h
        fp, gp, _ = evaluate("B", params + e)
        fm, gm, _ = evaluate("B", params - e)
        assert abs((fp - fm) / (2 * h) - grad[j]) < 1e-6 * max(1.0, abs(grad[j]))
        fd_col = (gp - gm) / (2 * h)
        assert np.allclose(fd_col, hess.reshape(5, 5)[:, j], rtol=1e-5, atol=1e-6)
