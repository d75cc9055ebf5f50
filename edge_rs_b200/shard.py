"""Gene sharding across ranks (one process per GPU).

Genes are independent (the reference fits them in a rayon par_iter and its
device path in independent searches), so the path shards by gene with no
exchange on the data path: every rank holds the design, offsets and subject
boundaries and fits a contiguous block of genes chosen so the blocks carry
about equal work, estimated per gene as (n_cells + nnz) x the evaluations its
search is expected to take: every sweep visits all cells plus the gene's
positive counts, and the search asks for about as many fits as evaluations.
Expected evaluations come from the caller (a previous fit's `evaluations`,
or the warm-start network's third output); without them every gene counts
the same. The only collective is the gather of the per-gene results at the
end (`torch.distributed.all_gather_object`, over NCCL or gloo).
"""
from typing import Callable, Optional

import numpy as np

from .api import NebulaError, NebulaFit


def shard_bounds(indptr, n_cells, world, evaluations=None):
    """Gene boundaries [b_0 = 0, ..., b_world = n_genes] of `world` contiguous
    blocks of about equal estimated work: (n_cells + nnz) per gene, times its
    expected `evaluations` when given (one per gene, positive)."""
    indptr = np.asarray(indptr, np.int64)
    n_genes = indptr.size - 1
    work = ((indptr[1:] - indptr[:-1]) + int(n_cells)).astype(np.float64)
    if evaluations is not None:
        ev = np.asarray(evaluations, np.float64)
        if ev.shape != (n_genes,):
            raise NebulaError(11, f"evaluations has {ev.size} entries, expected {n_genes}")
        work = work * np.where(np.isfinite(ev) & (ev > 0), ev, 1.0)
    cum = np.concatenate([[0], np.cumsum(work)])
    targets = cum[-1] * np.arange(world + 1) / world
    bounds = np.searchsorted(cum, targets, side="left")
    bounds[0], bounds[-1] = 0, n_genes
    return np.maximum.accumulate(bounds).astype(np.int64)


def slice_genes(counts, lo, hi):
    """Rows lo..hi of a gene-major CSR (indptr, indices, data, shape) as a CSR."""
    indptr, indices, data, shape = counts
    indptr = np.asarray(indptr)
    a, b = int(indptr[lo]), int(indptr[hi])
    sub_ptr = (indptr[lo:hi + 1] - a).astype(np.uint32)
    return (sub_ptr, np.asarray(indices)[a:b], np.asarray(data)[a:b], (hi - lo, shape[1]))


def merge_fits(parts, offsets, n_coef):
    """One NebulaFit from the ranks' fits; gene_index shifted by each block's first gene."""
    cat = lambda name: np.concatenate([getattr(p, name) for p in parts]) if parts else np.zeros(0)
    gene_index = np.concatenate([p.gene_index + off for p, off in zip(parts, offsets)]) if parts else np.zeros(0, int)
    stats = {}
    for p in parts:
        for k, v in p.stats.items():
            if isinstance(v, (int, float)):
                stats[k] = stats.get(k, 0) + v
    return NebulaFit(coefficients=cat("coefficients"), covariance=cat("covariance"), se=cat("se"),
                     subject_overdispersion=cat("subject_overdispersion"),
                     cell_overdispersion=cat("cell_overdispersion"), convergence=cat("convergence"),
                     sigma_at_bound=cat("sigma_at_bound"), gene_index=gene_index, n_coef=n_coef, stats=stats)


def fit_sharded(counts, subject_id, design, n_coef, offset=None, params=None, fit: Optional[Callable] = None,
                group=None, evaluations=None, **kwargs):
    """nebula_sparse_cuda over the ranks of torch.distributed's default (or
    given) group: each rank fits its block of genes on its own GPU (or with
    `fit`, any function of nebula_sparse_cuda's signature) and every rank
    returns the merged NebulaFit of all genes. evaluations: expected search
    evaluations per input gene, weighting the blocks (shard_bounds)."""
    import torch.distributed as dist
    if fit is None:
        from .api import nebula_sparse_cuda as fit
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    bounds = shard_bounds(counts[0], counts[3][1], world, evaluations)
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    mine = None
    if hi > lo:
        try:
            mine = fit(slice_genes(counts, lo, hi), subject_id, design, n_coef, offset, params, **kwargs)
        except NebulaError as e:
            if e.code != 7:  # NoGenesAfterFiltering: this block simply keeps no gene
                raise
    if world == 1:
        return merge_fits([mine] if mine is not None else [], [lo], n_coef)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    parts = [(g, int(bounds[r])) for r, g in enumerate(gathered) if g is not None]
    return merge_fits([p for p, _ in parts], [o for _, o in parts], n_coef)
