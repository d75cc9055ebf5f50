"""The opt_pml unit fixtures of src/sc/pml.rs:2149-2700 as arrays."""
import numpy as np

from golden_io import inline


def fixture(case):
    """(PmlData-like dict, n_beta) for one golden case."""
    G = inline()
    if case["fixture"] == "large":  # pml.rs:2610-2632
        starts = [0, 12, 32, 48, 64]
        design, offset, counts, cells, total = [], [], [], [], [0.0] * 4
        for i in range(64):
            design += [1.0, 1.0 if i % 3 == 0 else 0.0, (i % 7) / 8.0]
            offset.append(((i % 9) - 4.0) / 8.0)
            y = float((i * 7 + 3) % 11)
            if y > 0:
                counts.append(y)
                cells.append(i)
            s = min(max(j for j, b in enumerate(starts) if b <= i), 3)
            total[s] += y
        f = dict(design=design, offset=offset, counts=counts, cells=cells, subject_start=starts,
                 subject_total=total)
        return {k: np.asarray(v) for k, v in f.items()}, 3
    f = dict(G["pml_fixture_a"] if case["fixture"] == "A" else G["pml_fixture_b"])
    nb = 2
    if case.get("design") == "collinear":  # pml.rs:2474-2479
        d = np.array(f["design"]).reshape(12, 2)
        f["design"] = np.column_stack([d, d[:, 1]]).ravel()
        nb = 3
    elif case.get("design") == "ones":  # pml.rs:2504
        f["design"] = [1.0] * 12
        nb = 1
    return {k: np.asarray(v) for k, v in f.items()}, nb


def gene_view(work, g):
    """One gene of a synthetic workload in PmlData layout (centred design as NEBULA uses it)."""
    design = work["design_c"]
    lo, hi = int(work["indptr"][g]), int(work["indptr"][g + 1])
    cells = work["indices"][lo:hi]
    counts = work["data"][lo:hi]
    keep = counts > 0
    cells, counts = cells[keep], counts[keep]
    fid = work["fid"]
    subj_of = np.searchsorted(fid, cells, side="right") - 1
    total = np.bincount(subj_of, weights=counts, minlength=fid.size - 1)
    return dict(design=design, offset=work["log_offset"], counts=counts, cells=cells, subject_start=fid,
                subject_total=total)


def centred(design):
    """centre_design (ptmg.rs:1748-1797) for a design whose first column is the intercept."""
    out = design.astype(np.float64).copy()
    for j in range(design.shape[1]):
        col = design[:, j]
        mean = col.mean()
        sd = np.sqrt(((col - mean) ** 2).mean())
        out[:, j] = (col - mean) / sd if sd > 0 else 1.0
    return np.ascontiguousarray(out)
