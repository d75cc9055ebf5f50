"""Gene sharding across ranks (edge_rs_b200/shard.py): the balance of the
blocks, and a two-rank gloo run on the CPU whose gathered fit equals a
single-process fit gene for gene. The ranks fit with the FP64 oracle, which
stands in for each rank's GPU here; the sharding and the gather are the code
under test."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shard_bounds_cover_all_genes_and_balance_the_work():
    from edge_rs_b200.shard import shard_bounds
    rng = np.random.default_rng(0)
    nnz = rng.integers(0, 5000, 1000)
    indptr = np.concatenate([[0], np.cumsum(nnz)])
    for world in (1, 2, 3, 8):
        b = shard_bounds(indptr, 2000, world)
        assert b[0] == 0 and b[-1] == 1000 and np.all(np.diff(b) >= 0) and b.size == world + 1
        work = np.array([(indptr[b[r + 1]] - indptr[b[r]]) + 2000 * (b[r + 1] - b[r]) for r in range(world)])
        assert work.max() <= work.mean() * 1.02 + 7000


def test_shard_bounds_weight_by_expected_evaluations():
    """(n_cells + nnz) x expected evaluations per gene: a block of genes whose
    searches take four times the evaluations gets a quarter of the genes."""
    from edge_rs_b200.shard import shard_bounds
    indptr = np.arange(0, 1001 * 100, 100)  # 1000 genes of 100 entries
    ev = np.ones(1000)
    ev[:500] = 4.0
    b = shard_bounds(indptr, 1000, 2, evaluations=ev)
    cost = 1100.0 * ev
    halves = [cost[b[0]:b[1]].sum(), cost[b[1]:b[2]].sum()]
    assert abs(halves[0] - halves[1]) <= cost.max()
    assert b[1] < 500  # the expensive genes are split off early
    assert np.array_equal(shard_bounds(indptr, 1000, 2), shard_bounds(indptr, 1000, 2, evaluations=np.ones(1000)))


def test_slice_genes_keeps_rows():
    from edge_rs_b200.shard import slice_genes
    indptr = np.array([0, 2, 2, 5], np.uint32)
    indices = np.array([1, 3, 0, 2, 4], np.uint32)
    data = np.arange(5.0)
    sub = slice_genes((indptr, indices, data, (3, 6)), 1, 3)
    assert sub[0].tolist() == [0, 0, 3] and sub[1].tolist() == [0, 2, 4] and sub[3] == (2, 6)


def _dataset():
    from edge_rs_b200 import workloads
    return workloads.make("c0", seed=5, n_genes=10, n_cells=600, n_subjects=6)


def _oracle_fit(counts, subject, design, n_coef, offset, params):
    import oracle_ffi as of
    return of.nebula_sparse(counts, subject, design, n_coef, offset, params, threads=2)[0]


def _rank_main(rank, port, out):
    sys.path.insert(0, HERE)
    from datetime import timedelta

    import torch.distributed as dist

    from edge_rs_b200 import NebulaParams
    from edge_rs_b200.shard import fit_sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=timedelta(seconds=120))
    try:
        w = _dataset()
        fit = fit_sharded(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"), fit=_oracle_fit)
        if rank == 0:
            np.savez(out, coefficients=fit.coefficients, subject=fit.subject_overdispersion,
                     cell=fit.cell_overdispersion, gene_index=fit.gene_index, covariance=fit.covariance)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_process():
    import torch.multiprocessing as mp

    from edge_rs_b200 import NebulaParams
    w = _dataset()
    whole = _oracle_fit(w.csr, w.subject, w.design, w.n_coef, w.offset, NebulaParams(method="HL"))
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "rank0.npz")
        mp.start_processes(_rank_main, args=(_free_port(), out), nprocs=2, join=True, start_method="spawn")
        got = np.load(out)
        assert np.array_equal(got["gene_index"], whole.gene_index)
        assert np.array_equal(got["coefficients"], whole.coefficients)
        assert np.array_equal(got["subject"], whole.subject_overdispersion)
        assert np.array_equal(got["cell"], whole.cell_overdispersion)
        assert np.array_equal(got["covariance"], whole.covariance)
