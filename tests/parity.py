"""Comparison helpers shared by the parity tests.

Neighbour-list parity follows the contract: lists must agree for every pair
except those whose FP64 criterion value min(r2, rp2)/crit lies within a
relative band of 1 (the radius boundary).  For a mismatching (i, j) the band
membership is recomputed here in FP64 from the inputs.
"""
from __future__ import annotations

import numpy as np


def rel_err_vec(a: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-row |a - ref| / |ref| for (n, 3) arrays (or |.| for (n,))."""
    if a.ndim == 1:
        return np.abs(a - ref) / np.maximum(np.abs(ref), 1e-300)
    num = np.sqrt(((a - ref) ** 2).sum(1))
    den = np.sqrt((ref ** 2).sum(1))
    return num / np.maximum(den, 1e-300)


def list_rows(lst: np.ndarray):
    """Yield (nnb, ids) per row of a gpunb list array."""
    for row in lst:
        n = int(row[0])
        yield n, (row[1:1 + n] if n > 0 else row[1:1])


def criterion_ratio(i: int, j: int, mj, xj, vj, h2, dtr, xi, vi, m_flag: int) -> float:
    dx = xj[j] - xi[i]
    dv = vj[j] - vi[i]
    r2 = float(dx @ dx)
    p = dx + dtr[i] * dv
    rp2 = float(p @ p)
    crit = mj[j] * h2[i] if m_flag else h2[i]
    return min(r2, rp2) / crit


def pair_contrib(i: int, j: int, mj, xj, vj, xi, vi):
    """FP64 (acc, jrk, pot) contribution of j on i (gpunb pair rule)."""
    dx = xj[j] - xi[i]
    dv = vj[j] - vi[i]
    r2 = float(dx @ dx)
    rinv2 = 1.0 / r2
    mr = mj[j] * np.sqrt(rinv2)
    mr3 = mr * rinv2
    al = -3.0 * float(dx @ dv) * rinv2
    return mr3 * dx, mr3 * (dv + al * dx), mr


def align_to_lists(acc, jrk, pot, la, lb, inputs):
    """Return copies of (acc, jrk, pot) computed with list `la`, adjusted to
    what they would be with list `lb` (rows where neither overflowed): pairs
    that `lb` treats as neighbours are removed, pairs `la` treated as
    neighbours but `lb` does not are added.  This isolates arithmetic error
    from boundary-pair classification."""
    mj, xj, vj, xi, vi = inputs["mj"], inputs["xj"], inputs["vj"], inputs["xi"], inputs["vi"]
    acc, jrk, pot = acc.copy(), jrk.copy(), pot.copy()
    for i in range(la.shape[0]):
        na, nb_ = int(la[i, 0]), int(lb[i, 0])
        if na < 0 or nb_ < 0:
            continue
        sa = set(la[i, 1:1 + na].tolist())
        sb = set(lb[i, 1:1 + nb_].tolist())
        for j in sb - sa:   # lb excludes j, la included it
            a, jk, p = pair_contrib(i, j, mj, xj, vj, xi, vi)
            acc[i] -= a
            jrk[i] -= jk
            pot[i] -= p
        for j in sa - sb:   # la excluded j, lb includes it
            a, jk, p = pair_contrib(i, j, mj, xj, vj, xi, vi)
            acc[i] += a
            jrk[i] += jk
            pot[i] += p
    return acc, jrk, pot


def compare_lists(la: np.ndarray, lb: np.ndarray, inputs: dict, band: float,
                  m_flag: int = 0, max_straddle: int = 3) -> dict:
    """Compare two gpunb list arrays.  Returns counts of mismatching pairs
    inside/outside the boundary band and row-level count disagreements."""
    mj, xj, vj = inputs["mj"], inputs["xj"], inputs["vj"]
    h2, dtr, xi, vi = inputs["h2"], inputs["dtr"], inputs["xi"], inputs["vi"]
    cap = min(int(inputs["nnbmax"]), int(inputs["lmax"]) - 1) if "nnbmax" in inputs else 1 << 30
    out = {"rows": la.shape[0], "overflow_mismatch": 0, "overflow_straddle": 0,
           "pairs_in_band": 0,
           "pairs_out_of_band": 0, "worst_ratio_dev": 0.0, "checked_rows": 0,
           "unsorted_rows": 0}
    for i in range(la.shape[0]):
        na, nb_ = int(la[i, 0]), int(lb[i, 0])
        if (na < 0) != (nb_ < 0):
            # One side overflowed.  Acceptable only when the two counts
            # straddle the cap by a few boundary pairs.
            lo, hi = sorted((abs(na), abs(nb_)))
            if hi - lo <= max_straddle and lo <= cap < hi:
                out["overflow_straddle"] += 1
            else:
                out["overflow_mismatch"] += 1
            continue
        if na < 0:
            continue
        out["checked_rows"] += 1
        a = la[i, 1:1 + na]
        b = lb[i, 1:1 + nb_]
        if na > 1 and np.any(np.diff(a) <= 0):
            out["unsorted_rows"] += 1
        sa, sb = set(a.tolist()), set(b.tolist())
        for j in sa.symmetric_difference(sb):
            r = criterion_ratio(i, j, mj, xj, vj, h2, dtr, xi, vi, m_flag)
            dev = abs(r - 1.0)
            if dev <= band:
                out["pairs_in_band"] += 1
            else:
                out["pairs_out_of_band"] += 1
                out["worst_ratio_dev"] = max(out["worst_ratio_dev"], dev)
    return out
