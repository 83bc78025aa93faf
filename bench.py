#!/usr/bin/env python3
"""Benchmark of the trans/gw LMM association scan on B200.

Workload (seeded synthetic data with the benchmark shapes; no data set ships
with the reference): n = 2,000 samples (50 families of 10 siblings + 1,500
unrelated, founders' alleles at MAF ~ U(0.01, 0.5), 1% missing calls),
m = 500,000 SNPs, 10,000 genes with per-gene heritability h2 ~ U(0, 0.8) drawn
from the genotype covariance, intercept-only covariates; `--mode gw` (every
SNP against every gene). The metric counts tests = finite (SNP, gene) tests
(GeneSummary.n_tested), i.e. 5e9 per step.

One step = one pass of the path over the workload:
  value  genotypes decoded, phenotypes and the GRM eigenbasis resident in
         HBM: spectral rotation of all SNPs, per-gene REML prep, the
         tensor-core scan with its fused epilogue and the FP64 refinement of
         candidate pairs;
  e2e    the same job through the C ABI from HOST buffers: .bed bytes and
         phenotypes copied in, decode, GRM, eigendecomposition, rotation,
         REML, scan, refinement, results copied out.
Inputs are larger than L2 (the rotated genotypes alone are 8 GB), so no L2
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "trans-LMM SNP-gene tests/s, split-BF16 vs plain FP32 on 1 B200 at |Δlog10p|≤1e-3"
UNIT = "tests/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


def workload(args, seed_offset=0):
    from eqtl_b200 import synth
    t0 = time.time()
    rows, sub, _ = synth.make_bed_rows_chunked(20261208 + seed_offset, args.n, args.m, family=args.family,
                                               maf_lo=0.01, maf_hi=0.5, miss_rate=0.01,
                                               keep_codes_every=max(1, args.m // 2000))
    Y, _ = synth.polygenic_pheno(20261209 + seed_offset, sub, args.genes)
    X = np.ones((args.n, 1))
    return rows, Y, X, time.time() - t0


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def event_pair(ctx):
    import torch
    s = torch.cuda.ExternalStream(ctx.stream_ptr(), device=torch.device("cuda", ctx.device))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return s, a, b


def pinned(a):
    """Copy of `a` in page-locked host memory (a numpy view of a pinned torch
    tensor), so host->device copies run at link speed."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
    out = t.numpy()  # the view's base holds the tensor
    out[...] = a
    return out


def run_value_step(ctx):
    """Genotypes, eigenbasis and phenotypes resident: rotation + REML + scan
    + refinement."""
    ctx.rotate()
    genes, pairs, cands, delta = ctx.scan_trans_lmm(None, None, pthr=1e-5)
    return int(genes["n_tested"].sum()), len(pairs)


def run_e2e_step(ctx, rows, n, Y, X):
    """Whole job from host buffers: bed + phenotypes in, results out."""
    ctx.load_bed(rows, n, np.arange(n, dtype=np.int32))
    ctx.pheno_load(Y, X)
    ctx.lmm_basis(outputs=False)
    genes, pairs, cands, delta = ctx.scan_trans_lmm(None, None, pthr=1e-5)
    return int(genes["n_tested"].sum()), genes, pairs


# ----------------------------------------------------------- reference arm
# The reference program is timed on two contiguous SNP subsets of the
# workload (all n samples, the first `ref_genes` genes): REF_SNPS_SETUP SNPs
# and `ref_snps` SNPs. Every run pays the same one-off work (reading the
# tables, the eigendecomposition of the n x n GRM, one REML fit per gene), so
# the difference of the two gives the marginal rate of the scan itself - the
# rate a full run of the workload (5e9 tests) proceeds at, where that one-off
# work is negligible. The setup-inclusive rate of the larger run is reported
# beside it.
REF_SNPS_SETUP = 1000


def reference_sample(args, rows, Y, tmp, n_snps=None):
    """Writes a bounded sample of the workload (all n samples, the first
    `n_snps` (default `ref_snps`) SNPs, the first `ref_genes` genes) as
    PLINK + TSV files."""
    from eqtl_b200 import synth
    ms, gs = min(n_snps or args.ref_snps, args.m), min(args.ref_genes, args.genes)
    pre = os.path.join(tmp, f"sample{ms}")
    with open(pre + ".fam", "w") as f:
        for i in range(args.n):
            f.write(f"S{i + 1:05d} S{i + 1:05d} 0 0 0 -9\n")
    with open(pre + ".bim", "w") as f:
        for s in range(ms):
            f.write(f"1\trs{s + 1}\t0\t{100 * (s + 1)}\tA\tG\n")
    with open(pre + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(np.ascontiguousarray(rows[:ms]).tobytes())
    synth.write_pheno(os.path.join(tmp, "pheno.tsv"), [f"S{i + 1:05d}" for i in range(args.n)],
                      [f"G{g + 1:05d}" for g in range(gs)], Y[:, :gs])
    return pre, ms, gs


def run_reference(exe, pre, tmp, threads):
    out = os.path.join(tmp, "out")
    t0 = time.perf_counter()
    r = subprocess.run([exe, "-b", pre, "-e", os.path.join(tmp, "pheno.tsv"), "--model", "lmm", "--mode", "gw",
                        "--pval-trans", "1e-5", "-t", str(threads), "-o", out], capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    tested = 0
    with open(out + ".lmm.gw.region.tsv") as f:
        next(f)
        for ln in f:
            tested += int(ln.split("\t")[3])
    return tested, dt


def marginal_rate(tested_small, t_small, tested, t):
    """Tests per second of the scan beyond the one-off work both runs share,
    and that one-off time (s)."""
    rate = (tested - tested_small) / max(t - t_small, 1e-9)
    return rate, max(t_small - tested_small / rate, 0.0)


def reference_arm(args):
    exe = os.path.join(ROOT, "oracle", "_ref", "eqtl")
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference"}
    if not os.path.exists(exe):
        print(json.dumps({**base, "unavailable": "oracle/_ref/eqtl not built (make -C oracle needs the reference "
                                                   "sources)"}))
        return
    threads = os.cpu_count() or 1
    rows, Y, X, _ = workload(args)
    tmp = tempfile.mkdtemp(prefix="eqtl_ref_")
    try:
        pre0, ms0, _ = reference_sample(args, rows, Y, tmp, REF_SNPS_SETUP)
        pre, ms, gs = reference_sample(args, rows, Y, tmp)
        # the small run is the warm-up and the measure of the one-off work
        tested0, t0 = run_reference(exe, pre0, tmp, threads)
        times, tested = [], 0
        for _ in range(args.steps):
            tested, dt = run_reference(exe, pre, tmp, threads)
            times.append(dt)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    t_step = statistics.mean(times)
    value, setup_s = marginal_rate(tested0, t0, tested, t_step)
    # a step is one run of the larger sample; ms_per_step is its scan part
    ms_step = 1e3 * (t_step - setup_s)
    sample = (f"reference eqtl (built from its sources) --model lmm --mode gw -t {threads}, n={args.n}, "
              f"{gs} genes: marginal rate between {ms0} SNPs ({tested0} tests, {t0:.1f} s) and {ms} SNPs "
              f"({tested} tests, {t_step:.1f} s mean of {args.steps} runs); one-off work (tables, GRM "
              f"eigendecomposition, REML per gene) {setup_s:.1f} s per run")
    print(json.dumps({**base, "value": value, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic",
                      "config": config(args),
                      "setup_s": setup_s, "setup_inclusive_tests_per_s": tested / t_step,
                      "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                       "sample": sample},
                      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def config(args):
    return {"workload": "trans/gw LMM scan (--model lmm --mode gw)", "n_samples": args.n, "n_snps": args.m,
            "n_genes": args.genes, "covariates": "intercept", "family_structure": list(args.family),
            "pthr": 1e-5, "l2": "inputs larger than L2 (8 GB rotated genotypes)",
            "parallelism": f"replicas x{args.gpus}"}


# ------------------------------------------------------- replicas (N > 1)
def max_over_ranks(values, device):
    """Element-wise maximum of per-rank timings over the process group (the
    slowest replica sets the step time)."""
    import torch
    import torch.distributed as tdist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def whole_job_rate(tests_per_rank, world, ms_per_step):
    """Tests per second of the whole job: every replica tests the same
    workload, the step lasts as long as the slowest replica."""
    return tests_per_rank * world / (ms_per_step / 1e3)


# ------------------------------------------------------------------ B200 arm
def b200_arm(args, rank, world, local_rank):
    import torch
    from eqtl_b200 import capi
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        import datetime
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    rows, Y, X, gen_s = workload(args)
    n = args.n
    pk, pk_kind = peaks()

    # host inputs staged in pinned memory, the phenotypes gene-major as the
    # reference's phenotype table holds them (one row per gene)
    rows, Y = pinned(rows), pinned(np.ascontiguousarray(Y.T)).T
    ctx = capi.Context(local_rank)
    h2d = rows.nbytes + Y.nbytes + X.nbytes
    # ---- e2e: full job from host buffers through the C ABI
    e2e_ms = []
    tests = 0
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tests, genes, pairs = run_e2e_step(ctx, rows, n, Y, X)
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
    d2h = genes.nbytes + pairs.nbytes
    setup = {k: ctx.stage_ms(k) for k in ("decode", "grm", "eigen")}

    # ---- value: resident genotypes + basis
    for _ in range(args.warmup):
        run_value_step(ctx)
    stream, ev0, ev1 = event_pair(ctx)
    launches0 = ctx.launch_count()
    scan_ms, stage = [], {k: [] for k in ("rotate", "prep", "scan", "refine")}
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            tests, _ = run_value_step(ctx)
            for k in stage:
                stage[k].append(ctx.stage_ms(k))
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    ms_total = ev0.elapsed_time(ev1)
    e2e_mean = statistics.mean(e2e_ms) if e2e_ms else 0.0
    ms_total, e2e_mean = max_over_ranks([ms_total, e2e_mean], "cuda") if dist else (ms_total, e2e_mean)
    ms_step = ms_total / args.steps
    value = whole_job_rate(tests, world, ms_step)
    e2e_value = whole_job_rate(tests, world, e2e_mean) if e2e_ms else None

    # ---- roofline of the dominant kernel (the scan tile kernel)
    scan_ms = statistics.mean(stage["scan"])
    p_cov = X.shape[1]
    nodes, kcols = ctx.lmm_form()
    # issued tensor products per test: NUM from the exact SNP operand and a
    # split gene side (2 over K = n); gg and a_k either directly (gg from the
    # split Gt^2 and w: 3, each a_k like NUM: 2, over n) or interpolated
    # between node deltas (3 each over K = kcols node columns)
    issued = 2 * n * 2 + (2 * kcols * 3 * (p_cov + 1) if nodes else 2 * n * (3 + 2 * p_cov))
    form = f"gg and a_k interpolated between {nodes} node deltas (K = {kcols})" if nodes else "direct (K = n)"
    flops = tests * 2.0 * n * (p_cov + 2)
    achieved = flops / (scan_ms / 1e3) / 1e12
    peak = pk.get("bf16_tflops_sustained", FALLBACK_PEAKS["bf16_tflops_sustained"])
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": scan_traffic(tests), "kernel": "tile_kernel<128,3> (trans-LMM scan)",
            "algorithmic_flops_per_test": 2 * n * (p_cov + 2),
            "peak_source": f"{pk_kind} bf16 dense sustained (kernel runs under the power cap)",
            "issued_flops_per_test": issued, "form": form}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f16x2 split (FP32 accumulate), FP64 REML/refine", "data": "synthetic",
           "config": config(args),
           "stage_ms": {k: statistics.mean(v) for k, v in stage.items()}, "setup_ms": setup,
           "tests_per_step": tests, "gen_s": gen_s,
           "roofline": roof, "gpu_launches": launches,
           "clocks": clk.summary(),
           "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": e2e_mean if e2e_ms else None,
                   "ms_steps": [round(v, 1) for v in e2e_ms],
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}}

    # ---- plain FP32 CUDA-core comparator of the same scan (scan kernel only)
    if rank == 0 and not args.no_fp32:
        ctx32 = capi.Context(local_rank, precision=capi.PREC_FP32_SIMT)
        ctx32.load_bed(rows, n, np.arange(n, dtype=np.int32))
        ctx32.pheno_load(Y, X)
        ctx32.lmm_basis()
        run_value_step(ctx32)
        s32 = ctx32.stage_ms("scan")
        # FP32 CUDA-core peak at the clock sampled during the timed region:
        # 148 SMs x 128 FP32 lanes x 2 flops per FMA
        mhz = out["clocks"].get("sm_mhz") or 1965.0
        fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
        out["fp32_simt"] = {"scan_ms": s32, "tests_per_s_scan": tests / (s32 / 1e3),
                            "tensor_speedup": s32 / scan_ms,
                            "algorithmic_tflops": flops / (s32 / 1e3) / 1e12,
                            "fp32_peak_tflops_at_sampled_clock": fp32_peak,
                            "frac_of_fp32_peak": flops / (s32 / 1e3) / 1e12 / fp32_peak,
                            "form": "direct (gg and a_k over K = n)"}
        ctx32.close()
    # ---- the split-BF16 form of the same scan (BF16 hi + lo on both sides,
    # three products per accumulator: the exact dosage slice is FP16-only)
    if rank == 0 and not args.no_bf16:
        ctxb = capi.Context(local_rank, precision=capi.PREC_SPLIT_BF16)
        ctxb.load_bed(rows, n, np.arange(n, dtype=np.int32))
        ctxb.pheno_load(Y, X)
        ctxb.lmm_basis()
        run_value_step(ctxb)  # builds the BF16 SNP operands once
        sb = []
        for _ in range(3):
            run_value_step(ctxb)
            sb.append(ctxb.stage_ms("scan"))
        s16 = statistics.median(sb)
        out["bf16_split"] = {"scan_ms": s16, "tests_per_s_scan": tests / (s16 / 1e3),
                             "algorithmic_tflops": flops / (s16 / 1e3) / 1e12,
                             "frac": flops / (s16 / 1e3) / 1e12 / peak,
                             "issued_flops_per_test": 2 * n * 3 * (p_cov + 2),
                             "scan_ms_vs_f16": s16 / scan_ms}
        ctxb.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, rows, Y)
    ctx.close()
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def scan_traffic(tests):
    """DRAM bytes of the scan kernel per launch, scaled by the tests of a launch
    from the committed ncu capture of a smaller case (the SNP operand streams
    once per fixed-size gene group, so traffic grows with the tests):
    profiles/tile_kernel_lmm_scan_n2000_m100k_g4000.md, 'dram_bytes_per_test'."""
    p = os.path.join(ROOT, "profiles", "tile_kernel_lmm_scan_n2000_m100k_g4000.md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith("dram_bytes_per_test:"):
            return float(ln.split(":")[1]) * tests
    return None


def cpu_baseline(args, rows, Y):
    exe = os.path.join(ROOT, "oracle", "_ref", "eqtl")
    if not os.path.exists(exe):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "oracle/_ref not built"}
    threads = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="eqtl_cpu_")
    try:
        pre0, ms0, _ = reference_sample(args, rows, Y, tmp, REF_SNPS_SETUP)
        pre, ms, gs = reference_sample(args, rows, Y, tmp)
        tested0, t0 = run_reference(exe, pre0, tmp, threads)
        tested, dt = run_reference(exe, pre, tmp, threads)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    rate, setup_s = marginal_rate(tested0, t0, tested, dt)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
            "setup_inclusive_tests_per_s": tested / dt, "setup_s": setup_s,
            "sample": f"reference eqtl -t {threads}, n={args.n}, {gs} genes: marginal rate between {ms0} SNPs "
                      f"({t0:.1f} s) and {ms} SNPs ({tested} tests, {dt:.1f} s); one-off work (tables, GRM "
                      f"eigendecomposition, REML per gene) {setup_s:.1f} s per run"}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--m", type=int, default=500_000)
    ap.add_argument("--genes", type=int, default=10_000)
    ap.add_argument("--ref-snps", type=int, default=4000)
    ap.add_argument("--ref-genes", type=int, default=1000)
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-bf16", action="store_true", help="skip the split-BF16 form of the scan")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.family = (50, 10, args.n - 500) if args.n > 500 else None
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        return
    b200_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
