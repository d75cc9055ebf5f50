"""The learned warm start: training data from plain fits, GPU training with the
library's own kernels, and export of the built-in network.

The network (csrc/host/mlp_layout.hpp) maps 12 summary features of a gene
(log mean and log variance of its counts, zero fraction, per-subject spread,
stage one's sigma and gamma, ...) to the log-ratios of the final stage-two
(sigma, gamma) to stage one's and to the log number of stage-two objective
evaluations. `nebula_sparse_cuda(..., warm_start=True)` starts each gene's
search at the predicted point and finishes with the unchanged plain optimiser,
posts the genes predicted to need the most evaluations first, and refits an
audit sample cold.

Training data are plain (cold-start) fits of synthetic genes from NEBULA's
generative model (workloads.py), with sigma^2 and phi drawn LogNormal with sd
0.5 (the benchmark's draw) and 1.0 (wide) in alternate workloads, over a
spread of cell and subject counts.

Run on a GPU:  python -m edge_rs_b200.warm_start --out DIR
(writes DIR/warm_start_params.npy, DIR/warm_start_weights.inc, DIR/report.json)
"""
import argparse
import json
import os
import time

import numpy as np

from . import workloads
from ._ffi import MLP_FEATURES, MLP_OUTPUTS, MLP_PARAMS
from .api import NebulaParams, Session, mlp_init, mlp_train

# (cells, subjects) of the training workloads; 4-column design as c1
SHAPES = [(20000, 10), (20000, 40), (50000, 20), (50000, 64), (100000, 20), (100000, 100), (200000, 40)]


def examples(session, fit):
    """(features, targets) of a plain fit's searched genes."""
    feats, stage_one = session.features()
    ev = fit.evaluations.astype(np.float64)
    sigma = fit.subject_overdispersion
    gamma = 1.0 / fit.cell_overdispersion
    ok = (ev > 0) & np.isfinite(sigma) & np.isfinite(gamma) & (sigma > 0) & (gamma > 0) & (fit.convergence == 1)
    t = np.column_stack([np.log(sigma / stage_one[:, 0]), np.log(gamma / stage_one[:, 1]), np.log(np.maximum(ev, 1))])
    return feats[ok], t[ok].astype(np.float32)


def training_set(n_workloads=28, genes=600, seed=100):
    """Plain HL fits of synthetic workloads; returns (features, targets)."""
    xs, ts = [], []
    for i in range(n_workloads):
        n_cells, n_subj = SHAPES[i % len(SHAPES)]
        sd = 1.0 if (i // len(SHAPES)) % 2 else 0.5
        w = workloads.make("c1", seed=seed + i, n_genes=genes, n_cells=n_cells, n_subjects=n_subj,
                           sigma_log_sd=sd, phi_log_sd=sd)
        s = Session(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"))
        fit = s.fit()
        x, t = examples(s, fit)
        s.close()
        xs.append(x)
        ts.append(t)
    return np.concatenate(xs), np.concatenate(ts)


def train(features, targets, epochs=300, batch=512, lr=1e-3, seed=0):
    """A network with the features' normalisation, trained on the GPU."""
    params = mlp_init(seed)
    mean = features.mean(axis=0)
    sd = features.std(axis=0)
    params[MLP_PARAMS - 2 * MLP_FEATURES: MLP_PARAMS - MLP_FEATURES] = mean
    params[MLP_PARAMS - MLP_FEATURES:] = 1.0 / np.where(sd > 1e-6, sd, 1.0)
    return mlp_train(features, targets, params, epochs=epochs, batch=batch, lr=lr, seed=seed)


def export_inc(params, path):
    """Writes the built-in parameters as the C initializer warm_start.cpp includes."""
    p = np.asarray(params, np.float32)
    assert p.size == MLP_PARAMS
    head = ["// Generated by edge_rs_b200/warm_start.py; do not edit. The built-in warm-start",
            "// network's parameters (csrc/host/mlp_layout.hpp layout), trained on the GPU by",
            "// nb_mlp_train_cuda on plain fits of synthetic genes."]
    vals = [float.hex(float(v)) for v in p]
    rows = [", ".join(vals[i:i + 6]) + "," for i in range(0, len(vals), 6)]
    with open(path, "w") as fh:
        fh.write("\n".join(head + rows) + "\n")


def compare(params, name="c1", seed=1000, genes=500, n_cells=None, n_subjects=None):
    """Plain vs warm-started fits of one held-out workload: step time,
    evaluations and the largest differences of sigma and phi."""
    w = workloads.make(name, seed=seed, n_genes=genes, n_cells=n_cells, n_subjects=n_subjects)
    out = {}
    fits = {}
    for mode in (0, 1, 2):
        points = None
        if mode == 2:  # the plain fit's own optimum: the best a start can do
            points = np.ones((w.n_genes, 2))
            points[fits[0].gene_index, 0] = fits[0].subject_overdispersion
            points[fits[0].gene_index, 1] = 1.0 / fits[0].cell_overdispersion
        s = Session(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"), warm_start=mode,
                    mlp_weights=params if mode == 1 else None, warm_points=points)
        for _ in range(4):  # the cluster autotuner settles in the first calls
            s.fit()
        ms = []
        for _ in range(3):
            f = s.fit()
            ms.append(f.stats["ms_step_device"])
        s.close()
        fits[mode] = f
        out[("plain", "warm", "oracle_start")[mode]] = {"ms": float(np.median(ms)), "evaluations": int(f.evaluations.sum()),
                                            "requests": int(f.stats["requests"]), "sweeps": int(f.stats["sweeps"]),
                                            "audited": int(f.stats["audited"]),
                                            "refit_cold": int(f.stats["refit_cold"])}
    a, b = fits[0], fits[1]
    rel = lambda x, y: float(np.max(np.abs(x - y) / np.maximum(np.abs(x), 1e-12)))
    out["max_rel_diff"] = {"subject_overdispersion": rel(a.subject_overdispersion, b.subject_overdispersion),
                           "cell_overdispersion": rel(a.cell_overdispersion, b.cell_overdispersion),
                           "coefficients": rel(a.coefficients, b.coefficients)}
    out["speedup"] = out["plain"]["ms"] / out["warm"]["ms"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--workloads", type=int, default=28)
    ap.add_argument("--genes", type=int, default=600)
    ap.add_argument("--epochs", type=int, default=300)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    t0 = time.time()
    x, t = training_set(args.workloads, args.genes)
    t_data = time.time() - t0
    rng = np.random.default_rng(0)
    order = rng.permutation(len(x))
    hold = order[: len(x) // 10]
    fit_rows = order[len(x) // 10:]
    t1 = time.time()
    params, losses = train(x[fit_rows], t[fit_rows], epochs=args.epochs)
    t_train = time.time() - t1
    from .api import mlp_predict
    pred = mlp_predict(params, x[hold])
    base = np.zeros_like(t[hold])
    base[:, 2] = t[fit_rows, 2].mean()
    rmse = lambda p: np.sqrt(((p - t[hold]) ** 2).mean(axis=0)).tolist()
    np.save(os.path.join(args.out, "warm_start_params.npy"), params)
    export_inc(params, os.path.join(args.out, "warm_start_weights.inc"))
    report = {"examples": int(len(x)), "seconds_data": t_data, "seconds_train": t_train,
              "loss_first_last": [float(losses[0]), float(losses[-1])],
              "holdout_rmse": rmse(pred), "holdout_rmse_stage_one_start": rmse(base),
              "c1": compare(params)}
    with open(os.path.join(args.out, "report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
