"""Timings of the association-scan path at the benchmark shapes other than the
headline trans-LMM one (bench.py), through the C ABI with the inputs resident
on the device.

    python -m eqtl_b200.config_bench [--which grm,lm,glm] [--steps K]

grm  GRM build, eigendecomposition and spectral rotation: n = 2,000 samples
     (50 families of 10 siblings + 1,500 unrelated), m = 200,000 SNPs with
     MAF ~ U(0.01, 0.5) and 1% missing calls.
lm   trans/gw LM scan: n = 1,000 samples, m = 1,000,000 SNPs, 20,000 genes
     with Y ~ N(0, 1), intercept + 10 N(0, 1) covariates, p threshold 1e-5.
glm  gw NB-GLM scan: n = 1,000 samples, m = 200,000 SNPs, 5,000 genes of
     negative-binomial counts (synth.make_pheno_counts), intercept + 2
     covariates, p threshold 1e-5.
fission  PEER factors (15) of a 500 x 20,000 count table, and the
     rank-based inverse normal transform of the same table.

Seeded synthetic data of those shapes (no data set ships with the
reference). Each JSON line gives the CUDA-event stage times (median over the
timed steps, after one warm-up step) and the algorithmic rate of each stage's
dominant kernel against the measured peaks (the fallback figures when
MEASURED_PEAKS.json is absent).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics

import numpy as np

from . import capi, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def grm_case(steps: int) -> dict:
    n, m = 2000, 200_000
    rows, _, _ = synth.make_bed_rows_chunked(20261202, n, m, family=(50, 10, 1500), maf_lo=0.01, maf_hi=0.5,
                                             miss_rate=0.01)
    pk, kind = _peaks()
    with capi.Context(0) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        decode = c.stage_ms("decode")
        t = {"grm": [], "eigen": [], "rotate": []}
        for i in range(steps + 1):
            c.lmm_basis(outputs=False)
            c.rotate()
            if i:
                for k in t:
                    t[k].append(c.stage_ms(k))
    med = {k: statistics.median(v) for k, v in t.items()}
    m_kept = int(np.count_nonzero(keep))
    grm_flops = float(n) * (n + 1) * m_kept          # SYRK, symmetric half counted once
    rot_flops = 2.0 * n * n * m_kept
    peak = pk.get("bf16_tflops", 1590.0)
    return {"workload": "GRM build + eigendecomposition + spectral rotation", "n_samples": n, "n_snps": m,
            "kept_snps": m_kept, "steps": steps, "decode_ms": decode, "stage_ms": med, "stage_ms_steps": t,
            "grm": {"algorithmic_tflops": grm_flops / (med["grm"] / 1e3) / 1e12,
                    "frac_of_bf16_peak": grm_flops / (med["grm"] / 1e3) / 1e12 / peak,
                    "note": "stage time: per-SNP statistics, FP16 operand transpose, tensor-core SYRK "
                            "(lower-triangle tiles, 3 split products + missing-mask product), division"},
            "rotation": {"algorithmic_tflops": rot_flops / (med["rotate"] / 1e3) / 1e12,
                         "frac_of_bf16_peak": rot_flops / (med["rotate"] / 1e3) / 1e12 / peak},
            "peak_tflops": peak, "peak_source": kind, "data": "synthetic"}


def lm_case(steps: int, m: int = 1_000_000, G: int = 20_000) -> dict:
    n, ncov = 1000, 10
    rows, _, _ = synth.make_bed_rows_chunked(20261203, n, m, maf_lo=0.01, maf_hi=0.5, miss_rate=0.01)
    rng = np.random.default_rng(20261204)
    Y = rng.standard_normal((n, G))
    X = np.column_stack([np.ones(n), rng.standard_normal((n, ncov))])
    pk, kind = _peaks()
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        c.pheno_load(Y, X)
        t = {"prep": [], "scan": [], "refine": []}
        tests = 0
        for i in range(steps + 1):
            genes, pairs, _ = c.scan_trans_lm(None, None, pthr=1e-5)
            if i:
                tests = int(genes["n_tested"].sum())
                for k in t:
                    t[k].append(c.stage_ms(k))
    med = {k: statistics.median(v) for k, v in t.items()}
    step_ms = sum(med.values())
    flops = 2.0 * n * tests                               # numerators G~'Y_s
    peak = pk.get("bf16_tflops_sustained", 1400.0)
    return {"workload": "trans/gw LM scan (--model lm --mode gw)", "n_samples": n, "n_snps": m, "n_genes": G,
            "covariates": ncov, "pthr": 1e-5, "steps": steps, "tests_per_step": tests, "stage_ms": med,
            "stage_ms_steps": t,
            "tests_per_s": tests / (step_ms / 1e3), "pairs": int(len(pairs)),
            "scan": {"algorithmic_tflops": flops / (med["scan"] / 1e3) / 1e12,
                     "frac_of_bf16_sustained": flops / (med["scan"] / 1e3) / 1e12 / peak,
                     "issued_products": 2},  # y hi and lo against the exact dosage slice
            "peak_tflops": peak, "peak_source": kind, "data": "synthetic"}


def glm_case(steps: int, m: int = 200_000, G: int = 5_000) -> dict:
    n, ncov = 1000, 2
    rows, _, _ = synth.make_bed_rows_chunked(20261205, n, m, maf_lo=0.01, maf_hi=0.5, miss_rate=0.01)
    Y, C = synth.make_pheno_counts(20261206, None, G, ncov, n=n)
    X = np.column_stack([np.ones(n), C])
    pk, kind = _peaks()
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        c.pheno_load(Y, X)
        t = {"prep": [], "scan": [], "refine": []}
        tests = 0
        for i in range(steps + 1):
            genes, pairs, _, phi, conv = c.scan_glm(None, None, pthr=1e-5)
            if i:
                tests = int(genes["n_tested"].sum())
                for k in t:
                    t[k].append(c.stage_ms(k))
    med = {k: statistics.median(v) for k, v in t.items()}
    step_ms = sum(med.values())
    flops = 2.0 * n * (X.shape[1] + 2) * tests
    peak = pk.get("bf16_tflops_sustained", 1400.0)
    return {"workload": "gw NB-GLM scan (--model glm --mode gw)", "n_samples": n, "n_snps": m, "n_genes": G,
            "covariates": ncov, "pthr": 1e-5, "steps": steps, "tests_per_step": tests, "stage_ms": med,
            "stage_ms_steps": t, "tests_per_s": tests / (step_ms / 1e3), "pairs": int(len(pairs)),
            "converged": int(conv.sum()), "phi_median": float(np.median(phi)),
            "scan": {"algorithmic_tflops": flops / (med["scan"] / 1e3) / 1e12,
                     "frac_of_bf16_sustained": flops / (med["scan"] / 1e3) / 1e12 / peak,
                     "issued_products": 3},
            "peak_tflops": peak, "peak_source": kind, "data": "synthetic"}


def fission_case(steps: int, n: int = 500, G: int = 20_000, k: int = 15) -> dict:
    """PEER on the device (eqtl_peer) for a thinned count table of n samples
    x G genes with k factors and the reference's defaults (tol 1e-3, at most
    1000 iterations), from the reference's N(0, 1) starting values."""
    import time
    rng = np.random.default_rng(20261207)
    Y, _ = synth.make_pheno_counts(20261208, None, G, 0, n=n)
    X0 = rng.standard_normal((n, k))
    W0 = rng.standard_normal((G, k))
    times, iters = [], 0
    with capi.Context(0) as c:
        for i in range(steps + 1):
            t0 = time.perf_counter()
            _, iters = c.peer(Y, k, 1000, 1e-3, X0, W0)
            if i:
                times.append(1e3 * (time.perf_counter() - t0))
        t_int = []
        for i in range(steps + 1):
            t0 = time.perf_counter()
            c.pheno_int(Y)
            if i:
                t_int.append(1e3 * (time.perf_counter() - t0))
    return {"workload": "fission PEER + --pheno-norm int", "n_samples": n, "n_genes": G, "factors": k,
            "peer_iterations": iters, "peer_ms_steps": times, "peer_ms": statistics.median(times),
            "int_ms_steps": t_int, "int_ms": statistics.median(t_int),
            "note": "wall time of the C-ABI calls from host buffers (upload, device work, download)",
            "data": "synthetic"}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--which", default="grm,lm")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--lm-snps", type=int, default=1_000_000, help="SNPs of the lm case (smaller for profiling)")
    ap.add_argument("--lm-genes", type=int, default=20_000, help="genes of the lm case")
    ap.add_argument("--glm-snps", type=int, default=200_000, help="SNPs of the glm case (smaller for profiling)")
    ap.add_argument("--glm-genes", type=int, default=5_000, help="genes of the glm case")
    args = ap.parse_args()
    for w in args.which.split(","):
        if w == "grm":
            out = grm_case(args.steps)
        elif w == "glm":
            out = glm_case(args.steps, args.glm_snps, args.glm_genes)
        elif w == "fission":
            out = fission_case(args.steps)
        else:
            out = lm_case(args.steps, args.lm_snps, args.lm_genes)
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
