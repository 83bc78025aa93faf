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
