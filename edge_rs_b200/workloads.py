"""Seeded synthetic NEBULA workloads with the shapes of the benchmark configurations.

No public dataset backs the benchmark, so counts are drawn from NEBULA's own
generative model:

    y_gc ~ NB(mean = mu_gc * exp(b_gs), size = 1 / phi_g),  b_gs ~ N(0, sigma2_g)
    mu_gc = exp(x_c' beta_g) * lib_c / 2000,                lib_c ~ LogNormal(ln 2000, 0.3)

and the offset handed to NEBULA is lib_c, so the fitted intercept absorbs
-ln 2000. With an intercept of N(-2, 1) about 88% of entries are zero.
sigma2_g ~ LogNormal(ln 0.2, 0.5) and phi_g ~ LogNormal(ln 0.5, 0.5) (the
warm-start training set widens both log-sds to 1.0). Effects of non-intercept
columns are N(0, 0.5) on 10% of genes and zero elsewhere. Subject-level
columns are constant within a subject; cell-level covariates are N(0, 1).
Counts are stored as gene-major CSR (uint32 indptr/indices, float64 data).
"""
from dataclasses import dataclass
from typing import Optional

import numpy as np

CONFIGS = {
    # 200 genes x 5,000 cells, 10 subjects of 500, intercept + subject-level condition
    "c0": dict(n_genes=200, n_cells=5000, n_subjects=10, sizes="equal", n_subject_bin=1, n_cell_cov=0,
               batch=False, intercept=("normal", -2.0, 1.0)),
    # 500 genes x 100,000 cells, 20 subjects Dirichlet(2) sizes (min 500),
    # intercept, subject-level binary, cell covariate, subject-level batch
    "c1": dict(n_genes=500, n_cells=100000, n_subjects=20, sizes="dirichlet", n_subject_bin=1, n_cell_cov=1,
               batch=True, intercept=("normal", -2.0, 1.0)),
    # 4,000 genes x 50,000 cells, 64 subjects of 100-5,000 cells (log-uniform),
    # intercept, 2 subject-level binaries, 5 cell covariates, intercept U(-6, 1)
    "c2": dict(n_genes=4000, n_cells=50000, n_subjects=64, sizes="loguniform", n_subject_bin=2, n_cell_cov=5,
               batch=False, intercept=("uniform", -6.0, 1.0)),
    # 2,000 genes x 200,000 cells, 40 subjects, design as c2
    "c3": dict(n_genes=2000, n_cells=200000, n_subjects=40, sizes="loguniform", n_subject_bin=2, n_cell_cov=5,
               batch=False, intercept=("uniform", -6.0, 1.0)),
    # 20,000 genes x 100,000 cells, 100 subjects, 4 columns as c1
    "c4": dict(n_genes=20000, n_cells=100000, n_subjects=100, sizes="dirichlet", n_subject_bin=1, n_cell_cov=1,
               batch=True, intercept=("normal", -2.0, 1.0)),
}


@dataclass
class Workload:
    name: str
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    n_genes: int
    n_cells: int
    subject: np.ndarray
    design: np.ndarray
    offset: np.ndarray
    truth: dict

    @property
    def csr(self):
        return (self.indptr, self.indices, self.data, (self.n_genes, self.n_cells))

    @property
    def n_coef(self):
        return self.design.shape[1]

    @property
    def nnz(self):
        return int(self.data.size)


def subject_sizes(rng, n_cells, n_subjects, kind):
    if kind == "equal":
        sizes = np.full(n_subjects, n_cells // n_subjects)
    elif kind == "dirichlet":
        floor = min(500, n_cells // (2 * n_subjects))
        w = rng.dirichlet(np.full(n_subjects, 2.0))
        sizes = floor + np.floor(w * (n_cells - floor * n_subjects)).astype(np.int64)
    elif kind == "loguniform":
        raw = np.exp(rng.uniform(np.log(100.0), np.log(5000.0), n_subjects))
        sizes = np.maximum(1, np.floor(raw / raw.sum() * n_cells)).astype(np.int64)
    else:
        raise ValueError(kind)
    sizes = sizes.astype(np.int64)
    sizes[np.argmax(sizes)] += n_cells - sizes.sum()
    assert sizes.min() > 0 and sizes.sum() == n_cells
    return sizes


def make(name="c1", seed=0, n_genes: Optional[int] = None, n_cells: Optional[int] = None,
         n_subjects: Optional[int] = None, sigma_log_sd=0.5, phi_log_sd=0.5, chunk=64,
         gene_seed: Optional[int] = None):
    """Draws one workload; the named configuration may be shrunk for tests.
    gene_seed: draw the genes from their own stream (the cells, subjects and
    design still from `seed`), so that workloads drawn with one seed and
    different gene seeds share their cells and can be concatenated."""
    cfg = dict(CONFIGS[name])
    G = n_genes or cfg["n_genes"]
    N = n_cells or cfg["n_cells"]
    K = n_subjects or cfg["n_subjects"]
    rng = np.random.default_rng(seed)
    sizes = subject_sizes(rng, N, K, cfg["sizes"])
    subject = np.repeat(np.arange(K), sizes)
    cols = [np.ones(N)]
    for _ in range(cfg["n_subject_bin"]):  # balanced subject-level binaries
        level = np.zeros(K)
        level[rng.permutation(K)[: K // 2]] = 1.0
        cols.append(level[subject])
    for _ in range(cfg["n_cell_cov"]):
        cols.append(rng.standard_normal(N))
    if cfg["batch"]:
        level = np.zeros(K)
        level[rng.permutation(K)[: K // 2]] = 1.0
        cols.append(level[subject])
    design = np.column_stack(cols)
    p = design.shape[1]
    lib = np.exp(rng.normal(np.log(2000.0), 0.3, N))
    if gene_seed is not None:
        rng = np.random.default_rng([seed, gene_seed])
    kind, a, b = cfg["intercept"]
    intercept = rng.normal(a, b, G) if kind == "normal" else rng.uniform(a, b, G)
    beta = np.zeros((G, p))
    beta[:, 0] = intercept
    for j in range(1, p):
        on = rng.random(G) < 0.1
        beta[on, j] = rng.normal(0.0, 0.5, on.sum())
    sigma2 = np.exp(rng.normal(np.log(0.2), sigma_log_sd, G))
    phi = np.exp(rng.normal(np.log(0.5), phi_log_sd, G))
    b_subj = rng.standard_normal((G, K)) * np.sqrt(sigma2)[:, None]
    log_base = np.log(lib / 2000.0)
    indptr = np.zeros(G + 1, dtype=np.uint64)
    idx_parts, val_parts = [], []
    total = 0
    for g0 in range(0, G, chunk):
        g1 = min(G, g0 + chunk)
        eta = beta[g0:g1] @ design.T + log_base[None, :] + b_subj[g0:g1][:, subject]
        mean = np.exp(eta)
        size = (1.0 / phi[g0:g1])[:, None]
        lam = rng.gamma(size, mean / size)
        y = rng.poisson(lam).astype(np.float64)
        for r in range(g1 - g0):
            nz = np.flatnonzero(y[r])
            idx_parts.append(nz.astype(np.uint32))
            val_parts.append(y[r, nz])
            total += nz.size
            indptr[g0 + r + 1] = total
    if total >= 2 ** 32:
        raise ValueError("more stored counts than a uint32 CSR can index")
    indices = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.uint32)
    data = np.concatenate(val_parts) if val_parts else np.zeros(0)
    return Workload(name=name, indptr=indptr.astype(np.uint32), indices=indices, data=data, n_genes=G,
                    n_cells=N, subject=subject.astype(np.uint64), design=np.ascontiguousarray(design),
                    offset=lib, truth=dict(beta=beta, sigma2=sigma2, phi=phi, sizes=sizes))


def _draw(spec):
    """make(**spec) in a worker process."""
    return make(**spec)


def concat(parts):
    """One workload from parts that share their cells (drawn with one seed and
    different gene seeds): their genes stacked."""
    ptr = [np.asarray(parts[0].indptr, np.uint64)]
    for w in parts[1:]:
        ptr.append(np.asarray(w.indptr[1:], np.uint64) + ptr[-1][-1])
    indptr = np.concatenate(ptr)
    if indptr[-1] >= 2 ** 32:
        raise ValueError("more stored counts than a uint32 CSR can index")
    first = parts[0]
    return Workload(name=first.name, indptr=indptr.astype(np.uint32),
                    indices=np.concatenate([w.indices for w in parts]),
                    data=np.concatenate([w.data for w in parts]), n_genes=sum(w.n_genes for w in parts),
                    n_cells=first.n_cells, subject=first.subject, design=first.design, offset=first.offset,
                    truth=dict(sizes=first.truth["sizes"], sigma2=np.concatenate([w.truth["sigma2"] for w in parts]),
                               phi=np.concatenate([w.truth["phi"] for w in parts])))


def make_blocks(name, seed, n_genes=None, block=4000, procs=None):
    """A workload of the named configuration drawn in gene blocks of `block`
    in spawned worker processes (every block shares the cells, subjects and
    design of `seed`; block i draws its genes from gene seed i). For the
    largest configurations, where one process would take minutes."""
    import multiprocessing as mp
    import os
    G = n_genes or CONFIGS[name]["n_genes"]
    specs = [dict(name=name, seed=seed, n_genes=min(block, G - at), gene_seed=i)
             for i, at in enumerate(range(0, G, block))]
    procs = procs or max(1, min(16, os.cpu_count() or 1, len(specs)))
    with mp.get_context("spawn").Pool(procs) as pool:
        return concat(pool.map(_draw, specs))
