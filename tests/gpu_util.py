"""Shared helpers for the GPU parity tests."""
from __future__ import annotations

import math

import numpy as np

import restate as R


def acat_p_from(gene_res):
    """acat_p exactly as AcatAcc::p (src/stats_extra.cpp:24-31) from the
    device's tan sum / used count (long double arithmetic)."""
    out = np.ones(len(gene_res))
    for g, r in enumerate(gene_res):
        if r["acat_used"] == 0:
            continue
        T = np.longdouble(r["acat_tan_sum"]) / np.longdouble(int(r["acat_used"]))
        ac = 0.5 - float(np.arctan(T) / R._PI_L)
        out[g] = min(max(ac, 0.0), 1.0)
    return out


def log10_diff(a, b):
    a = np.maximum(np.asarray(a, float), 1e-300)
    b = np.maximum(np.asarray(b, float), 1e-300)
    return np.abs(np.log10(a) - np.log10(b))


# Stated absolute error of the device t statistic used by the screening
# epilogue, per contraction precision (FP32 accumulation in both): hi/lo
# FP16 keeps ~22 significant bits of every operand, hi/lo BF16 ~16. acat_p
# is checked against |dlog10 acat / dt| * T_ERR on top of the 1e-3 log10
# tolerance; pairs and best SNPs are FP64-refined and need no such term.
T_ERRS = {0: 2e-6, 1: 6.4e-5}
T_ERR = T_ERRS[0]


def check_scan(res, ora, pairs_ref, pthr, df, t_err=T_ERR, rel=1e-9):
    """rel: relative tolerance of the FP64-refined beta / t (1e-9 for LM; the
    LMM's REML delta comes from a different FP64 optimiser run, ~1e-8)."""
    genes, pairs, _ = res
    assert np.array_equal(genes["n_tested"], ora["n_tested"])
    ap = acat_p_from(genes)
    tol = 1e-3 + 3 * ora["acat_sens"] * t_err
    bad = log10_diff(ap, ora["acat_p"]) > tol
    assert not bad.any(), (np.nonzero(bad)[0][:5], ap[bad][:5], ora["acat_p"][bad][:5])
    got = {(int(q["snp"]), int(q["gene"])): q for q in pairs}
    # pair sets: identical except pairs whose p is within tolerance of pthr
    for k in set(got) ^ set(pairs_ref):
        pv = got[k]["p"] if k in got else pairs_ref[k]["p"]
        assert abs(np.log10(pv) - np.log10(pthr)) < 1e-6, (k, pv)
    for k in set(got) & set(pairs_ref):
        q, r = got[k], pairs_ref[k]
        assert abs(q["beta"] - r["beta"]) <= rel * abs(r["beta"]) + 1e-12, (k, q["beta"], r["beta"], q["t"], r["stat"])
        assert abs(q["t"] - r["stat"]) <= 10 * rel * abs(r["stat"]) + 1e-10, (k, q["t"], r["stat"])
        assert log10_diff(q["p"], r["p"]) < max(1e-8, 100 * rel)
    # best SNP per gene: identical, or a near-tie in p
    for gi in range(len(genes)):
        if ora["best_snp"][gi] < 0:
            assert genes["best_snp"][gi] == -1
            continue
        if genes["best_snp"][gi] != ora["best_snp"][gi]:
            pg = ora["stats"]["p"][genes["best_snp"][gi], gi]
            assert log10_diff(pg, ora["best_p"][gi]) < 1e-4
        assert log10_diff(genes["best_p"][gi], ora["best_p"][gi]) < 1e-4
