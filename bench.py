"""Benchmark of NEBULA-HL stage two on B200: genes/s at 100k cells.

Workload: 500 genes x 100,000 cells, 20 subjects (Dirichlet(2) sizes, min 500),
4-column design (intercept, subject-level binary, cell covariate, subject-level
batch), seeded synthetic counts from NEBULA's generative model, forced HL.

A step fits every gene of the workload. Two arms run on the same inputs: the
plain method (the reference's algorithm, bit-identical to the FP64 oracle;
`plain`) and the warm-started batched form the metric names (`value`): the
learned search start, a narrowed initial BOBYQA trust radius (3% of NLopt's)
and warm inner fits, 5% of the genes audited cold
(`--warm 0` makes the headline plain).
- `value`: stages two and three (every inner fit on the GPU) on inputs already
  resident in HBM (nb_session_fit), device time from CUDA events recorded on the
  library's launching stream around the step; L2 is flushed between steps.
- `e2e`: the drop-in nebula_sparse_cuda call from host buffers (validation,
  upload, stage one, stages two and three, download).
- `roofline`: the fit kernel against the measured FP64 FMA peak of this GPU
  (its work is FP64 arithmetic; neither HBM nor the tensor cores bound it).
- `cpu_baseline`: the FP64 CPU oracle (the reference's nebula_sparse restated)
  on a bounded gene sample of the same workload, all host threads.

`--impl reference` times that CPU path alone on the same workload and metric.
Multi-GPU (torchrun): weak scaling through the product's sharding: one
workload of N x 500 genes cut into blocks of equal estimated work
(edge_rs_b200/shard.py); each rank times its block, and the e2e leg calls
fit_sharded, whose only collective is the gather of the results.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from edge_rs_b200 import NebulaParams, workloads  # noqa: E402

METRIC = "NEBULA-HL genes/s @100k cells, 1 B200: warm-start+batched vs plain; roofline %"
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "fit_kernel_traffic.json")


def flops_per_visit(nv, sparse=False):
    """FP64 FLOP of one cell visit of the fit kernel's sweep (pml_fit_impl.cuh,
    sweep_sums with the table exp/log of nbmath.hpp), counted from the code:
    an FMA counts two, any other FP64 arithmetic instruction one; compares,
    integer and bit operations are not counted. nv: the design columns that
    vary within subjects (the others' shares are applied per subject).

    eta: the offset plus the subject's constant share (1) and nv FMAs (2 nv)
    exp (nb_exp_tab): 20 = x/L and the shifter (2), n (1), the two-part
        reduction (2 FMA), the degree-5 polynomial (3 FMA), q (3), the table
        product (3), the scale (1)
    t = e + gamma (1)
    log (nb_log_tab): 22 = r (1 FMA), the degree-7 polynomial (5 FMA), l1p (3),
        the exponent (1), hi and lo (2 FMA), their sum (2)
    1/t, correctly rounded (1), u = e/t (1)
    fold: resid and weight (2), per varying column the X'd FMA, p x and its
        sum (4 nv), the p x x' triangle (nv (nv + 1))
    a dense (zero-count) cell: sum log t (1), d = -gamma u (1), p = gamma u/t (2)
    a positive entry: log w_s in eta (1), sum y eta and sum y log t (2 FMA),
        d = y (1 - u) (2), p = y u/t (2)
    """
    common = 1 + 2 * nv + 20 + 1 + 22 + 1 + 1 + 2 + 4 * nv + nv * (nv + 1)
    return common + (9 if sparse else 4)


def varying_columns(design, subject):
    """How many design columns take more than one value within some subject
    (the reference's cell_level_columns, ptmg.rs:1962-2005)."""
    order = np.argsort(subject, kind="stable")
    x, sid = design[order], subject[order]
    starts = np.flatnonzero(np.r_[True, sid[1:] != sid[:-1]])
    lo = np.minimum.reduceat(x, starts, axis=0)
    hi = np.maximum.reduceat(x, starts, axis=0)
    return int(np.sum(np.any(lo != hi, axis=0)))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1")
    ap.add_argument("--genes", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per inner fit (0: the library's choice)")
    ap.add_argument("--warm", type=int, default=1,
                    help="warm start of the headline arm (0 plain, 1 learned start + warm inner fits)")
    ap.add_argument("--cpu-genes", type=int, default=32, help="gene sample of the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fit-batch", type=int, default=0,
                    help="instead of the bench: time launches of the fit kernel in batch mode, this many inner fits "
                         "of the workload's first gene per launch (the profiling workload)")
    ap.add_argument("--contraction", action="store_true",
                    help="instead of the bench: the Hessian contraction of config 3's final fits in FP64, FP32, "
                         "TF32 and split BF16 (tensor cores), with the errors it carries into se and log p")
    ap.add_argument("--zero-tables", action="store_true",
                    help="instead of the bench: the plain method on a categorical design (intercept and a "
                         "subject-level binary) of the default size, with the zero-count tables and with every "
                         "cell swept")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._thread = None

    def start(self):
        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([v.strip() for v in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()

    def stop(self):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 4 + i and r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        return world, rank, local, dist
    return 1, 0, local, None


def barrier_max(dist, value):
    """Max of a float over ranks (one all-reduce), or the value itself."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_sum(dist, value):
    """Sum of a float over ranks (one all-reduce), or the value itself."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_sample(work, n_genes):
    """The first n_genes genes of a workload as their own CSR."""
    n = min(n_genes, work.n_genes)
    end = int(work.indptr[n])
    return (work.indptr[: n + 1].copy(), work.indices[:end], work.data[:end], (n, work.n_cells))


def run_cpu(work, n_genes, threads):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi  # the oracle: checker and CPU baseline only
    csr = cpu_sample(work, n_genes)
    t0 = time.perf_counter()
    fit, _ = oracle_ffi.nebula_sparse(csr, work.subject, work.design, work.n_coef, work.offset,
                                      NebulaParams(method="HL"), threads=threads)
    el = time.perf_counter() - t0
    return len(fit.gene_index) / el, len(fit.gene_index), el, fit


def reference_arm(args, world, rank, dist):
    if rank != 0:
        return
    work = workloads.make(args.config, seed=1000, n_genes=args.genes)
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, n, el, _ = run_cpu(work, args.cpu_genes, threads)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "genes/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.cpu_genes / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded NEBULA generative model)",
            "config": {"workload": f"{args.config}: {work.n_genes} genes x {work.n_cells} cells, "
                                   f"{len(work.truth['sizes'])} subjects, {work.n_coef} columns, forced HL",
                       "sample_genes_per_step": args.cpu_genes},
            "cpu_baseline": {"value": value, "unit": "genes/s", "cores": threads, "kind": "port",
                             "sample": f"first {args.cpu_genes} genes of the workload per step"},
            "e2e": {"value": value, "unit": "genes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def l2_flush(buf):
    buf.add_(1.0)


def timed_session(args, work, params, flush, dist, warm, want_stage_one=False):
    """W warm-up and K timed nb_session_fit steps; L2 flushed before each.
    want_stage_one: also return stage one's (sigma, gamma) per kept gene."""
    import torch
    from edge_rs_b200.api import Session
    session = Session(work.csr, work.subject, work.design, work.n_coef, work.offset, params, cluster=args.cluster,
                      warm_start=warm)
    for _ in range(args.warmup):
        session.fit()
    step_ms, stats, t_wall, fit = [], [], 0.0, None
    for _ in range(args.steps):
        l2_flush(flush)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fit = session.fit()
        torch.cuda.synchronize()
        t_wall += time.perf_counter() - t0
        step_ms.append(fit.stats["ms_step_device"])
        stats.append(fit.stats)
    stage_one = session.features()[1] if want_stage_one else None
    session.close()
    return step_ms, stats, fit, t_wall, stage_one


def perturbed_plain(args, work, params, plain_fit, stage_one, delta):
    """The plain method with its search started from stage one's estimate
    times (1 + delta) for sigma and (1 - delta) for gamma: NLopt's trust
    radius, cold inner fits, no audit. Against the plain fit it measures how
    far two runs of the reference's search land apart from starts that
    differ by `delta` (the objective is flat to the search's resolution)."""
    from edge_rs_b200.api import Session
    points = np.zeros((work.n_genes, 2))
    points[plain_fit.gene_index, 0] = stage_one[:, 0] * (1.0 + delta)
    points[plain_fit.gene_index, 1] = stage_one[:, 1] * (1.0 - delta)
    s = Session(work.csr, work.subject, work.design, work.n_coef, work.offset, params, cluster=args.cluster,
                warm_start=2, warm_points=points, warm_radius=1.0, audit_percent=0, cold_inner=True)
    fit = s.fit()
    s.close()
    return fit


def rel_errors(a, b, eps):
    """Max and median of |a - b| / max(|a|, |b|) over the entries, an entry
    within eps absolute counting as zero (assert_relative_eq's semantics)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    if a.size == 0:
        return {"max": 0.0, "median": 0.0}
    diff = np.abs(a - b)
    scale = np.maximum(np.abs(a), np.abs(b))
    rel = np.where((diff <= eps) | (a == b), 0.0, diff / np.where(scale > 0, scale, 1.0))
    return {"max": float(np.max(rel)), "median": float(np.median(rel))}


def compare_fits(fit, ref):
    """Errors of `fit` against `ref` on the genes both kept: beta, sigma^2,
    phi (relative, eps 1e-9), Wald log p-values of every non-intercept
    coefficient (relative, eps 1e-6, as the parity tests), and how many
    convergence codes differ."""
    from edge_rs_b200 import glm_sc_test
    common = np.intersect1d(fit.gene_index, ref.gene_index)
    ia = np.searchsorted(fit.gene_index, common)
    ib = np.searchsorted(ref.gene_index, common)
    out = {"genes": int(common.size)}
    for key, name in (("coefficients", "beta"), ("subject_overdispersion", "sigma2"),
                      ("cell_overdispersion", "phi")):
        out[name] = rel_errors(getattr(fit, key)[ia], getattr(ref, key)[ib], 1e-9)
    la, lb = [], []
    for coef in range(1, fit.n_coef):
        la.append(glm_sc_test(fit.coefficients[ia], fit.covariance[ia], coef=coef).log_p_value)
        lb.append(glm_sc_test(ref.coefficients[ib], ref.covariance[ib], coef=coef).log_p_value)
    out["log_p"] = rel_errors(np.concatenate(la) if la else [], np.concatenate(lb) if lb else [], 1e-6)
    out["convergence_differs"] = int(np.sum(fit.convergence[ia] != ref.convergence[ib]))
    return out


def ours_arm(args, world, rank, local, dist):
    import torch
    from edge_rs_b200.api import measure_fp64_tflops, nebula_sparse_cuda
    torch.cuda.set_device(local)
    per_rank = args.genes or workloads.CONFIGS[args.config]["n_genes"]
    if per_rank * world > 4000:  # c4, or several ranks: gene blocks drawn in parallel
        full = workloads.make_blocks(args.config, seed=1000, n_genes=per_rank * world)
    else:
        full = workloads.make(args.config, seed=1000, n_genes=per_rank * world)
    work = full
    if world > 1:
        # weak scaling through the product's sharding: one workload of world x
        # the per-rank genes (the same draw on every rank), each rank fitting
        # the block shard_bounds gives it; the e2e leg calls fit_sharded
        from edge_rs_b200.shard import shard_bounds, slice_genes
        bounds = shard_bounds(full.indptr, full.n_cells, world)
        lo, hi = int(bounds[rank]), int(bounds[rank + 1])
        ptr, ind, dat, _ = slice_genes(full.csr, lo, hi)
        work = workloads.Workload(name=full.name, indptr=ptr, indices=ind, data=dat, n_genes=hi - lo,
                                  n_cells=full.n_cells, subject=full.subject, design=full.design,
                                  offset=full.offset, truth=full.truth)
    params = NebulaParams(method="HL")
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    # the plain method (the reference's algorithm, bit-identical to the oracle)
    plain_ms, plain_stats, plain_fit, _, stage_one = timed_session(args, work, params, flush, dist, 0,
                                                                   want_stage_one=True)
    plain_value = (all_sum(dist, len(plain_fit.gene_index)) * args.steps
                   / (barrier_max(dist, float(np.sum(plain_ms))) / 1000.0))
    # the headline: warm-started (learned search start, narrowed initial trust
    # radius, warm inner fits) and batched
    sampler = ClockSampler(local)
    sampler.start()
    step_ms, stats, fit, t_wall, _ = timed_session(args, work, params, flush, dist, args.warm)
    clocks = sampler.stop()
    genes = len(fit.gene_index)
    total_ms = barrier_max(dist, float(np.sum(step_ms)))
    value = all_sum(dist, genes) * args.steps / (total_ms / 1000.0)
    launches = int(np.sum([s["gpu_launches"] for s in stats]))
    visits = float(np.sum([s["cell_visits"] for s in stats]))
    sparse_visits = float(np.sum([s["sparse_visits"] for s in stats]))
    kernel_ms = float(np.sum([s["ms_device"] for s in stats]))
    fp64_peak = measure_fp64_tflops(5)
    # the fit kernel is the whole step (one persistent launch serves stages
    # two and three), so its FLOP are divided by the step's device time;
    # dense (zero-count) and positive visits are counted apart
    n_varying = varying_columns(work.design, work.subject)
    flop = ((visits - sparse_visits) * flops_per_visit(n_varying)
            + sparse_visits * flops_per_visit(n_varying, sparse=True))
    achieved = flop / (float(np.sum(step_ms)) / 1000.0) / 1e12
    # DRAM bytes of one launch, measured by ncu on the c1 workload of 500
    # genes (one pass over the whole persistent launch); no figure for other
    # workloads
    traffic = None
    if os.path.exists(PROFILE_SUMMARY) and args.config == "c1" and genes == 500 and world == 1:
        try:
            with open(PROFILE_SUMMARY) as fh:
                traffic = json.load(fh).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    # end to end through the drop-in C-ABI call from host buffers
    e2e_vals, h2d, d2h = [], 0, 0
    e2e_stats = {"ms_stage_one": None, "ms_stage_two": None, "ms_stage_three": None}
    e2e_all = []
    for _ in range(args.e2e_steps):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if world > 1:  # every rank returns the whole job's merged fit
            from edge_rs_b200.shard import fit_sharded
            f2 = fit_sharded(full.csr, full.subject, full.design, full.n_coef, full.offset, params,
                             cluster=args.cluster, warm_start=args.warm)
        else:
            f2 = nebula_sparse_cuda(work.csr, work.subject, work.design, work.n_coef, work.offset, params,
                                    cluster=args.cluster, warm_start=args.warm)
        torch.cuda.synchronize()
        el = barrier_max(dist, time.perf_counter() - t0)
        e2e_vals.append(len(f2.gene_index) / el)
        h2d = f2.stats["h2d_bytes"]
        d2h = f2.stats["d2h_bytes"]
        e2e_all.append(f2.stats)
    if e2e_vals:  # the breakdown of the median call
        e2e_stats = e2e_all[int(np.argsort(e2e_vals)[len(e2e_vals) // 2])]
    # the search's reproducibility floor: the plain method from starts
    # perturbed by 1e-9 and by 1e-3 relative
    floors = {f"plain_from_start_x(1+-{d:g})": perturbed_plain(args, work, params, plain_fit, stage_one, d)
              for d in (1e-9, 1e-3)}
    if rank != 0:
        return
    cpu, parity = None, None
    if world == 1 and not args.no_cpu_baseline:
        cv, n, el, ref = run_cpu(work, args.cpu_genes, os.cpu_count() or 1)
        cpu = {"value": cv, "unit": "genes/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"first {n} of the workload's genes ({el:.1f} s of CPU work)"}
        # every arm against the FP64 oracle on the sampled genes, at the
        # workload's full size
        parity = {"oracle_sample": f"first {n} genes of the workload, FP64 CPU oracle",
                  "plain": compare_fits(plain_fit, ref), "warm": compare_fits(fit, ref),
                  **{k: compare_fits(v, ref) for k, v in floors.items()}}
    vs_plain = {"warm": compare_fits(fit, plain_fit), **{k: compare_fits(v, plain_fit) for k, v in floors.items()}}
    line = {
        "metric": METRIC, "value": value, "unit": "genes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded NEBULA generative model; no public dataset)",
        "config": {"workload": f"{args.config}: {work.n_genes} genes x {work.n_cells} cells, "
                               f"{len(work.truth['sizes'])} subjects, {work.n_coef} columns, forced HL, "
                               + ("warm-started (learned search start, initial trust radius 3% of NLopt's, "
                                  "warm inner fits, 5% audited cold)"
                                  if args.warm else "plain cold start"),
                   "genes_per_rank": genes, "nnz_per_rank": work.nnz, "l2": "flushed (256 MiB write) before each step",
                   "step": "stages two and three on device-resident inputs (nb_session_fit)"},
        "plain": {"value": plain_value, "ms_per_step": float(np.sum(plain_ms)) / args.steps,
                  "sweeps_per_step": plain_stats[-1]["sweeps"], "requests_per_step": plain_stats[-1]["requests"],
                  "evaluations_per_gene": float(plain_fit.evaluations.mean())},
        "warm_vs_plain": value / plain_value,
        "warm_start": {"mode": args.warm, "audited": stats[-1]["audited"], "refit_cold": stats[-1]["refit_cold"],
                       "evaluations_per_gene": float(fit.evaluations.mean())},
        # max / median relative errors (beta, sigma^2, phi: eps 1e-9; Wald log p
        # of every non-intercept coefficient: eps 1e-6) and differing
        # convergence codes: each arm against the FP64 oracle on a gene sample,
        # and against the plain arm on every gene
        "parity": parity,
        "vs_plain_all_genes": vs_plain,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp64_peak if fp64_peak > 0 else None, "traffic": traffic,
                     "kernel": "fit_queue_kernel",
                     "flops_per_visit": {"dense": flops_per_visit(n_varying),
                                         "positive": flops_per_visit(n_varying, sparse=True)},
                     "visits_per_step": {"dense": (visits - sparse_visits) / args.steps,
                                         "positive": sparse_visits / args.steps},
                     "varying_columns": n_varying,
                     "flop_counting": "an FMA counts two, other FP64 arithmetic one (bench.py flops_per_visit)",
                     "time": "device time of the step (CUDA events around the persistent launch)",
                     "peak_source": "measured on this GPU: FP64 FMA chains (nb_measure_fp64_tflops)"},
        # the median call: the host's cores are shared with other jobs, and a
        # call that meets their load is slower in every phase at once
        "e2e": {"value": float(np.median(e2e_vals)) if e2e_vals else None, "unit": "genes/s",
                "statistic": f"median of {len(e2e_vals)} calls", "calls": [float(v) for v in e2e_vals],
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_total": e2e_stats.get("ms_total"),
                "ms_prepare": e2e_stats.get("ms_prepare"), "ms_upload": e2e_stats.get("ms_upload"),
                "ms_stage_one": e2e_stats["ms_stage_one"],
                "ms_stage_two": e2e_stats["ms_stage_two"], "ms_stage_three": e2e_stats["ms_stage_three"]},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "detail": {"rounds_per_step": stats[-1]["rounds"], "requests_per_step": stats[-1]["requests"],
                   "sweeps_per_step": stats[-1]["sweeps"], "cell_visits_per_step": stats[-1]["cell_visits"],
                   "kernel_ms_per_step": kernel_ms / args.steps, "wall_ms_per_step": 1000.0 * t_wall / args.steps,
                   # share of the fit CTAs' slot-time spent inside requests
                   "slot_utilisation": stats[-1]["slot_cycles"] / (stats[-1]["fit_slots"] * stats[-1]["ms_step_device"]
                                                                   * 1e-3 * clocks["sm_mhz"] * 1e6)
                   if clocks.get("sm_mhz") else None,
                   "cycles_per_visit_per_cta": stats[-1]["slot_cycles"] / stats[-1]["cell_visits"],
                   "ctas_per_fit": stats[-1]["cluster"], "fit_slots": stats[-1]["fit_slots"],
                   # device time from the first fit's start to the last fit's end, and
                   # the step's device time outside it (start-up and the drain)
                   "busy_span_ms": stats[-1]["ms_busy_span"],
                   # summed over the fits: device time clusters waited for their tickets
                   "ticket_wait_ms": stats[-1]["ms_ticket_wait"],
                   "outside_span_ms": stats[-1]["ms_step_device"] - stats[-1]["ms_busy_span"]},
    }
    print(json.dumps(line), flush=True)


def zero_tables(args):
    """The plain method (stages two and three on resident inputs, L2 flushed
    before each step) on a categorical design at the default workload's size,
    once with the zero-count tables and once with every cell swept. Prints one
    JSON line."""
    import torch
    from edge_rs_b200.api import Session
    base = workloads.CONFIGS[args.config]
    work = workloads.make("c0", seed=1000, n_genes=args.genes or base["n_genes"], n_cells=base["n_cells"],
                          n_subjects=base["n_subjects"])
    params = NebulaParams(method="HL")
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out, fits = {}, {}
    for name, dense in (("tables", False), ("dense", True)):
        s = Session(work.csr, work.subject, work.design, work.n_coef, work.offset, params, dense_sweep=dense)
        for _ in range(args.warmup):
            s.fit()
        ms = []
        for _ in range(args.steps):
            l2_flush(flush)
            torch.cuda.synchronize()
            f = s.fit()
            ms.append(f.stats["ms_step_device"])
        s.close()
        fits[name] = f
        out[name] = {"genes_per_s": len(f.gene_index) * args.steps / (float(np.sum(ms)) / 1000.0),
                     "ms_per_step": float(np.mean(ms)), "zero_groups": f.stats["zero_groups"],
                     "cell_visits_per_step": f.stats["cell_visits"], "sweeps_per_step": f.stats["sweeps"]}
    a, b = fits["tables"], fits["dense"]
    print(json.dumps({"mode": "zero-tables", "config": {"workload": f"c0 design: {work.n_genes} genes x "
                                                        f"{work.n_cells} cells, {len(work.truth['sizes'])} subjects, "
                                                        f"{work.n_coef} columns, forced HL, plain method"},
                      **out, "speedup": out["tables"]["genes_per_s"] / out["dense"]["genes_per_s"],
                      "tables_vs_dense": compare_fits(a, b)}), flush=True)


def contraction_study(args):
    """The inner fit's Hessian contraction at the workload's shape (default
    config 3: 200,000 cells, 40 subjects, 8 columns) in four arithmetics
    (nb_contract_krx_cuda): FP64 / FP32 on CUDA cores, TF32 / split BF16 on
    the tensor cores. The weights are those of each gene's final fit: the
    plain method fits up to 128 genes, the subjects' log w are solved at the
    fitted beta, sigma and phi, and w_c = (gamma + y_c) e_c / (e_c + gamma)^2.
    For each variant: the contraction's error against the FP64 one, the
    information matrix it gives (gamma S minus the subjects' Schur terms,
    those in FP64), and the errors that carries into the standard errors and
    the Wald log p-values; its device time and rate. Prints one JSON line."""
    import torch
    from edge_rs_b200 import glm_sc_test
    from edge_rs_b200.api import CONTRACT_VARIANTS, Session, contract_krx_cuda
    cfg = args.config if args.config != "c1" else "c3"
    n_genes = min(args.genes or 128, 128)
    work = workloads.make(cfg, seed=1000, n_genes=n_genes)
    s = Session(work.csr, work.subject, work.design, work.n_coef, work.offset, NebulaParams(method="HL"))
    fit = s.fit()
    s.close()
    dev = torch.device("cuda")
    kept = fit.gene_index
    R, N, p = len(kept), work.n_cells, work.n_coef
    X = torch.from_numpy(work.design).to(dev)
    subj = torch.from_numpy(work.subject.astype(np.int64)).to(dev)
    K = int(work.subject.max()) + 1
    Y = torch.zeros((R, N), dtype=torch.float64, device=dev)
    for r, g in enumerate(kept):
        lo, hi = int(work.indptr[g]), int(work.indptr[g + 1])
        Y[r, torch.from_numpy(work.indices[lo:hi].astype(np.int64)).to(dev)] = torch.from_numpy(work.data[lo:hi]).to(dev)
    beta = torch.from_numpy(fit.coefficients).to(dev)
    eta0 = beta @ X.T + torch.log(torch.from_numpy(work.offset).to(dev))[None, :]
    sig2 = torch.from_numpy(fit.subject_overdispersion).to(dev)[:, None]
    gam = (1.0 / torch.from_numpy(fit.cell_overdispersion).to(dev))[:, None]
    exps = 1.0 + sig2
    alpha, lam = 1.0 / (exps - 1.0), 1.0 / (torch.sqrt(exps) * (exps - 1.0))

    def seg(v):  # per-subject sums of an R x N array
        return torch.zeros((R, K), dtype=torch.float64, device=dev).index_add_(1, subj, v)

    lw = torch.zeros((R, K), dtype=torch.float64, device=dev)
    for _ in range(100):  # each subject's log w at the fitted beta (Newton on the penalised likelihood)
        e = torch.exp(eta0 + lw[:, subj])
        t = e + gam
        score = seg(Y - (Y + gam) * e / t) + alpha - lam * torch.exp(lw)
        curv = gam * seg((gam + Y) * e / (t * t)) + lam * torch.exp(lw)
        step = score / curv
        lw = lw + step
        if float(step.abs().max()) < 1e-14:
            break
    e = torch.exp(eta0 + lw[:, subj])
    t = e + gam
    W = (gam + Y) * e / (t * t)
    bounds = np.concatenate([[0], np.cumsum(work.truth["sizes"])])
    vwb = torch.stack([gam * (W[:, a:b] @ X[a:b]) for a, b in zip(bounds[:-1], bounds[1:])], dim=1)  # R x K x p
    vw = gam * seg(W) + lam * torch.exp(lw)
    schur = torch.einsum("rka,rkb->rab", vwb / vw[:, :, None], vwb)
    pairs = [(a, b) for b in range(p) for a in range(b + 1)]

    def information(S):
        full = torch.zeros((R, p, p), dtype=torch.float64, device=dev)
        for j, (a, b) in enumerate(pairs):
            full[:, a, b] = S[:, j]
            full[:, b, a] = S[:, j]
        return gam[:, :, None] * full - schur

    def wald(info):
        cov = torch.linalg.inv(info).cpu().numpy()
        packed = np.stack([cov[:, a, b] for a, b in pairs], axis=1)
        se = np.sqrt(np.stack([cov[:, j, j] for j in range(p)], axis=1))
        logp = np.stack([glm_sc_test(fit.coefficients, packed, coef=c).log_p_value for c in range(1, p)], axis=1)
        return packed, se, logp

    out = {}
    base = None
    ref_dgemm = None
    for v, name in CONTRACT_VARIANTS.items():
        ms = []
        for _ in range(args.warmup + args.steps):
            S, m_kernel, m_total = contract_krx_cuda(v, X, W)
            ms.append((m_kernel, m_total))
        m_kernel = float(np.median([a for a, _ in ms[args.warmup:]]))
        m_total = float(np.median([b for _, b in ms[args.warmup:]]))
        packed, se, logp = wald(information(S))
        se = se[:, 1:]  # the slopes: the intercept's se depends on the design's centring
        flop = 2.0 * R * N * len(pairs) * (3 if v == 3 else 1)
        entry = {"ms_kernel": m_kernel, "ms_with_conversions": m_total,
                 "tflops": flop / (m_kernel * 1e-3) / 1e12}
        if base is None:
            base = (S, se, logp)
            # sanity: FP64 against a cuBLAS DGEMM of the same product, and the
            # recomputed covariance against the fit's own
            kr = torch.stack([X[:, a] * X[:, b] for a, b in pairs], dim=1)
            ref_dgemm = W @ kr
            entry["vs_dgemm_max_rel"] = float(((S - ref_dgemm).abs() / ref_dgemm.abs().amax(1, keepdim=True)).max())
            # the slopes' variances (the fit reports the intercept's in centred
            # coordinates, these are in the design's own)
            diag = [b * (b + 1) // 2 + b for b in range(1, p)]
            entry["slope_variance_vs_fit"] = rel_errors(packed[:, diag], fit.covariance[:, diag], 0.0)
        else:
            S0, se0, logp0 = base
            entry["contraction_max_rel"] = float(((S - S0).abs() / S0.abs().amax(1, keepdim=True)).max())
            entry["se_slopes"] = rel_errors(se, se0, 0.0)
            entry["log_p"] = rel_errors(logp, logp0, 1e-6)
        out[name] = entry
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    print(json.dumps({"mode": "contraction", "config": {"workload": f"{cfg}: {R} genes' final fits x {N} cells, "
                                                                    f"{K} subjects, {p} columns ({len(pairs)} "
                                                                    "Khatri-Rao columns)"},
                      "variants": out, "measured_peaks": peaks,
                      "beta_sigma2_phi": "unchanged at the fit's fixed point: the contraction steers Newton "
                                         "only; the value, gradient and log-determinant stay FP64"}), flush=True)


def fit_batch(args):
    """R inner fits of one c1-shaped gene per launch through nb_opt_pml_cuda:
    the per-fit code of the persistent launch (fit_one) in the batch kernel,
    a bounded single launch for the profiler. Prints one JSON line."""
    from edge_rs_b200.api import opt_pml_cuda
    work = workloads.make(args.config, seed=1000, n_genes=1)
    lo, hi = int(work.indptr[0]), int(work.indptr[1])
    cells, counts = work.indices[lo:hi], work.data[lo:hi]
    keep = counts > 0
    cells, counts = cells[keep], counts[keep]
    fid = np.concatenate([[0], np.cumsum(work.truth["sizes"])]).astype(np.uint64)
    subj = np.searchsorted(fid, cells, side="right") - 1
    total = np.bincount(subj, weights=counts, minlength=fid.size - 1)
    design = work.design.astype(np.float64)
    log_off = np.log(work.offset)
    beta0 = np.zeros(work.n_coef)
    beta0[0] = np.log(max(counts.sum() / work.n_cells, 1e-3)) - float(np.mean(log_off))
    rng = np.random.default_rng(0)
    r = args.fit_batch
    sigma = rng.uniform(0.05, 1.5, r)
    gamma = np.exp(rng.uniform(np.log(0.5), np.log(10.0), r))
    times, sweeps = [], 0
    for _ in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = opt_pml_cuda(design, log_off, counts, cells, fid, total, beta0, sigma, gamma)
        times.append(time.perf_counter() - t0)
        sweeps = int(out["sweeps"].sum())
    ms = 1000.0 * float(np.median(times[args.warmup:]))
    print(json.dumps({"mode": "fit-batch", "requests": r, "n_cells": int(work.n_cells), "nnz": int(cells.size),
                      "sweeps_per_launch": sweeps, "ms_per_call": ms}), flush=True)


def main():
    args = parse()
    if args.fit_batch > 0:
        fit_batch(args)
        return
    if args.zero_tables:
        zero_tables(args)
        return
    if args.contraction:
        contraction_study(args)
        return
    if args.impl == "reference":  # rank 0 alone times the CPU path; other ranks exit
        reference_arm(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), None)
        return
    world, rank, local, dist = dist_setup(args)
    try:
        ours_arm(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
