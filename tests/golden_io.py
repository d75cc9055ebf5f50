"""Loaders for the committed golden fixtures (written by golden/make_goldens.py)."""
import csv
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "golden", "data")


def inline():
    with open(os.path.join(HERE, "golden", "inline_goldens.json")) as fh:
        return json.load(fh)


def _field(text):
    t = text.strip().strip('"')
    if t in ("NA", "NaN", "nan"):
        return float("nan")
    if t in ("Inf", "inf"):
        return float("inf")
    if t in ("-Inf", "-inf"):
        return float("-inf")
    return float(t)


def table(name):
    """A headed CSV as (column names, row-major float matrix)."""
    with open(os.path.join(DATA, name)) as fh:
        rows = [r for r in csv.reader(fh) if r]
    names = [n.strip().strip('"') for n in rows[0]]
    values = np.array([[_field(v) for v in r] for r in rows[1:]], dtype=np.float64)
    return names, values


def column(tbl, name):
    names, values = tbl
    return values[:, names.index(name)]


def dense_to_csr(dense):
    """Gene-major CSR of the strictly positive entries of a genes x cells matrix."""
    indptr = [0]
    indices, data = [], []
    for row in dense:
        nz = np.nonzero(row > 0)[0]
        indices.extend(nz.tolist())
        data.extend(row[nz].tolist())
        indptr.append(len(data))
    return (np.array(indptr, np.uint32), np.array(indices, np.uint32), np.array(data, np.float64),
            dense.shape)


# tests/e2e_nebula.rs:288-398: (method, has_offset, n_coef, design_file)
E2E = {
    "sc": ("LN", True, 3, False),
    "sc_small": ("LN", True, 3, False),
    "sc_k2": ("HL", True, 3, True),
    "sc_blocks": ("LN", True, 3, True),
    "sc_intercept": ("HL", False, 1, True),
    "sc_wide": ("HL", True, 8, True),
    "sc_high": ("HL", True, 3, True),
    "sc_xwide": ("LN", True, 13, True),
    "sc_cat_ln": ("LN", True, 4, True),
    "sc_cat_hl": ("HL", True, 4, True),
    "sc_cat_sparse": ("HL", True, 3, True),
}


def load_e2e(tag):
    """One end-to-end dataset (tests/e2e_nebula.rs:404-448)."""
    method, has_offset, n_coef, design_file = E2E[tag]
    _, counts = table(f"{tag}_counts.csv")
    meta = table(f"{tag}_meta.csv")
    subject = column(meta, "subject").astype(np.int64) - 1
    n_cells = counts.shape[1]
    if design_file:
        _, design = table(f"{tag}_design.csv")
    else:
        design = np.column_stack([np.ones(n_cells), column(meta, "grp"), column(meta, "cov2")])
    offset = column(meta, "offset") if has_offset else None
    return dict(tag=tag, method=method, counts=counts, csr=dense_to_csr(counts), subject=subject,
                design=np.ascontiguousarray(design, dtype=np.float64), n_coef=n_coef, offset=offset)


def expected_e2e(tag, n_coef):
    """R's nebula output for a dataset: coefficients, se, subject, cell, covariance (crate packing)."""
    want = table(f"{tag}_nebula.csv")
    names = want[0]
    coef_names = [n[len("logFC_"):] for n in names if n.startswith("logFC_")][:n_coef]
    coef = np.column_stack([column(want, f"logFC_{c}") for c in coef_names])
    se = np.column_stack([column(want, f"se_{c}") for c in coef_names])
    p = np.column_stack([column(want, f"p_{c}") for c in coef_names])
    cov_t = table(f"{tag}_covariance.csv")
    packed = n_coef * (n_coef + 1) // 2
    cov_r = np.column_stack([column(cov_t, f"cov_{k + 1}") for k in range(packed)])
    cov = np.zeros_like(cov_r)
    k = 0
    for j in range(n_coef):  # R's lower.tri column-major -> upper column-major (e2e_nebula.rs:509-530)
        for i in range(j, n_coef):
            cov[:, i * (i + 1) // 2 + j] = cov_r[:, k]
            k += 1
    algorithm = column(want, "algorithm") if "algorithm" in names else np.zeros(len(coef))
    return dict(gene_index=column(want, "gene_id").astype(np.int64) - 1, coef=coef, se=se, p=p,
                subject=column(want, "Subject"), cell=column(want, "Cell"),
                convergence=column(want, "convergence").astype(np.int64), cov=cov, algorithm=algorithm)


def load_eight_gene():
    """The 8 x 150 golden of src/sc/nebula.rs:2377-2393 (6 subjects of 25 cells -> HL)."""
    counts = np.loadtxt(os.path.join(DATA, "nebula_counts.csv"), delimiter=",", ndmin=2)
    _, raw = table("nebula_design.csv")
    subject = raw[:, 0].astype(np.int64)
    design = np.column_stack([np.ones(raw.shape[0]), raw[:, 1], raw[:, 2]])
    return dict(counts=counts, csr=dense_to_csr(counts), subject=subject, design=design, n_coef=3,
                offset=raw[:, 3].copy())


def expected_eight_gene():
    want = table("nebula_expected.csv")
    _, cov = table("nebula_covariance.csv")
    values = want[1]
    cov_crate = cov[:, [0, 1, 3, 2, 4, 5]]  # nebula.rs:2421-2423 repack
    return dict(coef=values[:, 0:3], se=values[:, 3:6], p=values[:, 6:9], subject=values[:, 10],
                cell=values[:, 11], convergence=values[:, 12].astype(np.int64), cov=cov_crate)


def close(got, want, max_relative, epsilon=0.0):
    """assert_relative_eq semantics: |a-b| <= eps or <= max_rel * max(|a|,|b|)."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    diff = np.abs(got - want)
    scale = np.maximum(np.abs(got), np.abs(want))
    ok = (diff <= epsilon) | (diff <= max_relative * scale) | (got == want)
    return bool(np.all(ok)), float(np.max(np.where(scale > 0, diff / np.where(scale > 0, scale, 1), 0.0)))
