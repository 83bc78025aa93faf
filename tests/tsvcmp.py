"""Comparison helpers for eqtl TSV outputs (pairs / top / region files).

Rows are keyed by (gene, snp) for pairs/top and by gene for region files, so
row order (which depends on thread count and on the SNP-outer vs gene-outer
path in the reference) does not matter. Numeric columns are compared with
explicit tolerances; text columns must be identical.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

PAIR_COLS = ["gene", "snp", "chrom", "pos", "ref", "alt", "af", "beta", "se", "stat", "p", "r2",
             "n", "tss_dist", "scope"]
REGION_COLS = ["gene", "chrom", "tss", "n_tested", "n_sig", "acat_p", "q_bh", "p_emp", "p_beta",
               "beta_shape1", "beta_shape2"]


def read_tsv(path: str) -> Tuple[List[str], List[List[str]]]:
    with open(path) as f:
        lines = f.read().splitlines()
    return lines[0].split("\t"), [ln.split("\t") for ln in lines[1:] if ln]


def _num(s: str) -> float:
    if s in ("NA", "nan", "-nan"):
        return float("nan")
    return float(s)


def log10p_diff(a: float, b: float) -> float:
    fa, fb = max(a, 1e-300), max(b, 1e-300)
    return abs(math.log10(fa) - math.log10(fb))


class Tol:
    def __init__(self, rel=1e-6, abs_=1e-9, log10p=1e-3, beta_rel=1e-4):
        self.rel, self.abs, self.log10p, self.beta_rel = rel, abs_, log10p, beta_rel


def close(a: float, b: float, rel: float, abs_: float) -> bool:
    if math.isnan(a) or math.isnan(b):
        return math.isnan(a) and math.isnan(b)
    return abs(a - b) <= abs_ + rel * max(abs(a), abs(b))


def compare_pairs(ref_rows: Sequence[Sequence[str]], got_rows: Sequence[Sequence[str]],
                  tol: Tol, p_thr: Optional[float] = None) -> List[str]:
    """Returns a list of human-readable mismatches (empty = equal). Pairs
    present on one side only are forgiven when their p is within tolerance of
    the threshold p_thr."""
    errs: List[str] = []
    R = {(r[0], r[1]): r for r in ref_rows}
    G = {(r[0], r[1]): r for r in got_rows}
    for k in set(R) ^ set(G):
        row = R.get(k) or G.get(k)
        p = _num(row[10])
        if p_thr is not None and log10p_diff(p, p_thr) <= 10 * tol.log10p:
            continue
        errs.append(f"pair {k} only in {'ref' if k in R else 'got'} (p={row[10]})")
    for k in set(R) & set(G):
        r, g = R[k], G[k]
        for i in (0, 1, 2, 3, 4, 5, 12, 13, 14):
            if i == 13 and r[i] != "NA":
                if not close(_num(r[i]), _num(g[i]), 0, 0.5):
                    errs.append(f"{k} tss_dist {r[i]} vs {g[i]}")
                continue
            if r[i] != g[i]:
                errs.append(f"{k} col {PAIR_COLS[i]}: {r[i]!r} vs {g[i]!r}")
        rp, gp = _num(r[10]), _num(g[10])
        if log10p_diff(rp, gp) > tol.log10p:
            errs.append(f"{k} p {r[10]} vs {g[10]}")
        rb, gb = _num(r[7]), _num(g[7])
        if not close(rb, gb, tol.beta_rel, tol.abs):
            errs.append(f"{k} beta {r[7]} vs {g[7]}")
        for i in (6, 8, 9, 11):
            if not close(_num(r[i]), _num(g[i]), tol.beta_rel, 1e-7):
                errs.append(f"{k} {PAIR_COLS[i]} {r[i]} vs {g[i]}")
        if len(r) != len(g):
            errs.append(f"{k} {len(r)} vs {len(g)} columns")
        elif len(r) == 17:                       # GLM: phi, glm_converged
            if not close(_num(r[15]), _num(g[15]), tol.beta_rel, 1e-9):
                errs.append(f"{k} phi {r[15]} vs {g[15]}")
            if r[16] != g[16]:
                errs.append(f"{k} glm_converged {r[16]} vs {g[16]}")
    return errs


def compare_region(ref_rows, got_rows, tol: Tol, check_perm=True, acat_sens=None,
                   t_err: float = 0.0) -> List[str]:
    """acat_sens: gene -> |d log10 acat_p / d t| from the oracle; the acat_p
    tolerance is tol.log10p + 3 * sens * t_err (t_err = the stated absolute
    error of every t statistic on the checked side). A gene's q_bh is the
    minimum of p * G / rank over the genes at or above its rank, a function
    of all the acat_p that moves (in log10) by at most the largest move of
    any acat_p: q_bh passes within its own gene's tolerance or within the
    largest acat_p difference of the file (each of which is checked
    against its own tolerance)."""
    errs: List[str] = []
    R = {r[0]: r for r in ref_rows}
    G = {r[0]: r for r in got_rows}
    for k in set(R) ^ set(G):
        errs.append(f"region gene {k} only in {'ref' if k in R else 'got'}")
    sens = acat_sens or {}
    d_max = 0.0
    for k in set(R) & set(G):
        a, b = _num(R[k][5]), _num(G[k][5])
        if not (math.isnan(a) or math.isnan(b)):
            d_max = max(d_max, log10p_diff(a, b))
    for k in set(R) & set(G):
        r, g = R[k], G[k]
        for i in (1, 2, 3, 4):
            if r[i] != g[i]:
                errs.append(f"{k} {REGION_COLS[i]}: {r[i]} vs {g[i]}")
        lim = tol.log10p + 3.0 * sens.get(k, 0.0) * t_err
        for i, li in ((5, lim), (6, max(lim, d_max + 1e-9))):
            a, b = _num(r[i]), _num(g[i])
            if math.isnan(a) != math.isnan(b) or (not math.isnan(a) and log10p_diff(a, b) > li):
                errs.append(f"{k} {REGION_COLS[i]}: {r[i]} vs {g[i]}")
        if check_perm:
            for i in (7,):
                a, b = _num(r[i]), _num(g[i])
                if not close(a, b, 1e-9, 1e-12):
                    errs.append(f"{k} {REGION_COLS[i]}: {r[i]} vs {g[i]}")
            for i in (8, 9, 10):
                a, b = _num(r[i]), _num(g[i])
                if not close(a, b, 5e-2, 1e-12):
                    errs.append(f"{k} {REGION_COLS[i]}: {r[i]} vs {g[i]}")
    return errs
