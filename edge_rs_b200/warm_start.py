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
generative model (workloads.py): 200,000 genes from config 2's generator
(50,000 cells, 64 subjects of 100-5,000 cells, 8 columns) with sigma^2 and
phi LogNormal sd 1.0, and 4-column workloads over a spread of cell and
subject counts with sd 0.5 (the benchmark's draw) and 1.0 alternating. The
network infers with BF16 weights and FP32 accumulation (nb_mlp_predict_cuda)
and is trained in FP32. The report evaluates it on a held-out c1 workload
and on config 4 (20,000 genes x 100,000 cells, 100 subjects).

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


_draw = workloads._draw


def _fits(specs, procs):
    """(features, targets) of plain fits of the workloads `specs` describe,
    drawn `procs` at a time in spawned worker processes."""
    import multiprocessing as mp
    xs, ts = [], []
    with mp.get_context("spawn").Pool(procs) as pool:
        for at in range(0, len(specs), procs):
            for w in pool.map(_draw, specs[at:at + procs]):
                s = Session(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"))
                x, t = examples(s, s.fit())
                s.close()
                xs.append(x)
                ts.append(t)
    return np.concatenate(xs), np.concatenate(ts)


def training_set(n_workloads=28, genes=600, seed=100, c2_genes=200000, c2_per_workload=4000, procs=None):
    """Plain HL fits of synthetic workloads; returns (features, targets):
    `c2_genes` genes from config 2's generator (50,000 cells, 64 subjects,
    8 columns) with sigma^2 and phi LogNormal sd 1.0, and n_workloads x genes
    genes of 4-column workloads over SHAPES (sd 0.5 and 1.0 alternating)."""
    procs = procs or max(1, min(16, os.cpu_count() or 1))
    specs = [dict(name="c2", seed=seed + 1000 + i, n_genes=c2_per_workload, sigma_log_sd=1.0, phi_log_sd=1.0)
             for i in range(c2_genes // c2_per_workload)]
    for i in range(n_workloads):
        n_cells, n_subj = SHAPES[i % len(SHAPES)]
        sd = 1.0 if (i // len(SHAPES)) % 2 else 0.5
        specs.append(dict(name="c1", seed=seed + i, n_genes=genes, n_cells=n_cells, n_subjects=n_subj,
                          sigma_log_sd=sd, phi_log_sd=sd))
    return _fits(specs, procs)


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


def compare(params, name="c1", seed=1000, genes=500, n_cells=None, n_subjects=None, work=None, steps=3,
            warmup=4):
    """Plain vs warm-started fits of one held-out workload (5% of the warm
    runs' genes audited cold): step time, evaluations and the differences
    from plain. Modes: plain; the learned start; stage one's start with the
    same warm inner fits and radius (what the network adds is the gap
    between these two); the plain fit's own optimum as the start (the best
    a start can do)."""
    w = work or workloads.make(name, seed=seed, n_genes=genes, n_cells=n_cells, n_subjects=n_subjects)
    out = {"workload": f"{w.name}: {w.n_genes} genes x {w.n_cells} cells, {len(w.truth['sizes'])} subjects, "
                       f"{w.n_coef} columns"}
    fits = {}
    for label, mode in (("plain", 0), ("learned_start", 1), ("stage_one_start", 3), ("optimum_start", 2)):
        points = None
        if mode == 2:
            points = np.ones((w.n_genes, 2))
            points[fits["plain"].gene_index, 0] = fits["plain"].subject_overdispersion
            points[fits["plain"].gene_index, 1] = 1.0 / fits["plain"].cell_overdispersion
        s = Session(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"), warm_start=mode,
                    mlp_weights=params if mode == 1 else None, warm_points=points)
        for _ in range(warmup):  # the cluster autotuner settles in the first calls
            s.fit()
        ms = []
        for _ in range(steps):
            f = s.fit()
            ms.append(f.stats["ms_step_device"])
        s.close()
        fits[label] = f
        out[label] = {"ms": float(np.median(ms)), "genes_per_s": len(f.gene_index) / (float(np.median(ms)) * 1e-3),
                      "evaluations": int(f.evaluations.sum()), "requests": int(f.stats["requests"]),
                      "sweeps": int(f.stats["sweeps"]), "audited": int(f.stats["audited"]),
                      "refit_cold": int(f.stats["refit_cold"])}
    a = fits["plain"]
    rel = lambda x, y: np.where(np.abs(x - y) <= 1e-9, 0.0, np.abs(x - y) / np.maximum(np.abs(x), np.abs(y)))
    for label in ("learned_start", "stage_one_start"):
        b = fits[label]
        out[label]["vs_plain"] = {k: {"max": float(rel(getattr(a, k), getattr(b, k)).max()),
                                      "q95": float(np.quantile(rel(getattr(a, k), getattr(b, k)), 0.95)),
                                      "median": float(np.median(rel(getattr(a, k), getattr(b, k))))}
                                  for k in ("subject_overdispersion", "cell_overdispersion", "coefficients")}
        out[label]["speedup_vs_plain"] = out["plain"]["ms"] / out[label]["ms"]
    out["learned_vs_stage_one_start"] = out["stage_one_start"]["ms"] / out["learned_start"]["ms"]
    return out


def config4(params, procs, parts=5, seed=4000):
    """Config 4's evaluation workload (20,000 genes x 100,000 cells, 100
    subjects, 4 columns) drawn in `parts` gene blocks in parallel."""
    work = workloads.make_blocks("c4", seed, block=workloads.CONFIGS["c4"]["n_genes"] // parts,
                                 procs=min(procs, parts))
    return compare(params, work=work, steps=2, warmup=2)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--workloads", type=int, default=28)
    ap.add_argument("--genes", type=int, default=600)
    ap.add_argument("--c2-genes", type=int, default=200000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--no-c4", action="store_true")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    procs = max(1, min(16, os.cpu_count() or 1))
    t0 = time.time()
    x, t = training_set(args.workloads, args.genes, c2_genes=args.c2_genes, procs=procs)
    t_data = time.time() - t0
    rng = np.random.default_rng(0)
    order = rng.permutation(len(x))
    hold = order[: len(x) // 10]
    fit_rows = order[len(x) // 10:]
    t1 = time.time()
    params, losses = train(x[fit_rows], t[fit_rows], epochs=args.epochs)
    t_train = time.time() - t1
    from .api import mlp_predict
    pred = mlp_predict(params, x[hold])  # BF16 weights, FP32 accumulation
    base = np.zeros_like(t[hold])
    base[:, 2] = t[fit_rows, 2].mean()
    rmse = lambda p: np.sqrt(((p - t[hold]) ** 2).mean(axis=0)).tolist()
    np.save(os.path.join(args.out, "warm_start_params.npy"), params)
    export_inc(params, os.path.join(args.out, "warm_start_weights.inc"))
    report = {"examples": int(len(x)), "c2_generator_genes": args.c2_genes, "epochs": args.epochs,
              "seconds_data": t_data, "seconds_train": t_train,
              "loss_first_last": [float(losses[0]), float(losses[-1])],
              "holdout_rmse_bf16_weights": rmse(pred), "holdout_rmse_stage_one_start": rmse(base),
              "c1": compare(params)}
    if not args.no_c4:
        report["c4"] = config4(params, procs)
    with open(os.path.join(args.out, "report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
