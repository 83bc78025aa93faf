"""Throughput of the cis permutation path through the eqtl program.

    python -m eqtl_b200.perm_bench [--genes G] [--perm B] [--models lmm,lm]
    python -m eqtl_b200.perm_bench --lognormal --genes 20000 --perm 1000 --models lmm

--lognormal gives the cis-LMM permutation benchmark's shape: 10 chromosomes
of 50 Mb whose SNP density is constant within each 2 Mb segment and drawn
lognormal across segments (median 1,500 per Mb, sd 0.9 on the log scale,
clamped to 25 - 7,500 per Mb), so that the +-1 Mb cis windows hold a
lognormal number of SNPs (median about 3,000, from about 50 to 15,000);
genes have uniform TSS over the genome. The realised window sizes are
reported (percentiles).

Seeded synthetic data with the shape of the cis-LMM permutation workload:
n = 1,000 samples (25 families of 10 siblings + 750 unrelated), 3 chromosomes
of 10 Mb at 1,500 SNPs per Mb (about 3,000 SNPs in each gene's +-1 Mb window),
15 N(0,1) covariates, G genes with polygenic phenotypes (h2 ~ U(0, 0.8)),
`--mode cis -w 1000000 --perm B`. Every permuted column gets its own REML fit
and its own banded cis scan, as in the reference. The program runs with
EQTL_TRACE=1; the JSON line reports wall time, the device stages of the
permutation scans (CUDA events) and permuted columns per second.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

from . import synth

PKG = os.path.dirname(os.path.abspath(__file__))


def make_case(d: str, genes: int, n: int = 1000, n_chrom: int = 3, chrom_mb: int = 10, per_mb: int = 1500,
              n_cov: int = 15) -> int:
    m = n_chrom * chrom_mb * per_mb
    fam = (25, 10, n - 250) if n > 250 else None
    rows, sub, _ = synth.make_bed_rows_chunked(4242, n, m, family=fam, keep_codes_every=20)
    rng = np.random.default_rng(7)
    clen = chrom_mb * 1_000_000
    chrom, pos = [], []
    for c in range(n_chrom):
        p = np.sort(rng.choice(np.arange(1, clen + 1), size=m // n_chrom, replace=False))
        chrom += [str(c + 1)] * (m // n_chrom)
        pos.append(p)
    pos = np.concatenate(pos)
    samples = [f"S{i + 1:05d}" for i in range(n)]
    pre = os.path.join(d, "geno")
    with open(pre + ".fam", "w") as f:
        for s in samples:
            f.write(f"{s} {s} 0 0 0 -9\n")
    with open(pre + ".bim", "w") as f:
        for i in range(m):
            f.write(f"{chrom[i]}\trs{i + 1}\t0\t{int(pos[i])}\tA\tG\n")
    with open(pre + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(rows.tobytes())
    Y, _ = synth.polygenic_pheno(11, sub, genes)
    C = rng.standard_normal((n, n_cov))
    Y += 0.5 * C.sum(1, keepdims=True)
    ids, gc, st, en, sd, _ = synth.make_genes(5, genes, [str(c + 1) for c in range(n_chrom)], clen, body=1)
    synth.write_pheno(os.path.join(d, "pheno.tsv"), samples, ids, Y)
    synth.write_covar(os.path.join(d, "covar.tsv"), samples, C)
    synth.write_gff(os.path.join(d, "genes.gff"), ids, gc, st, en, sd)
    return m


def make_case_lognormal(d: str, genes: int, n: int = 1000, n_chrom: int = 10, chrom_mb: int = 50,
                        n_cov: int = 15) -> int:
    rng = np.random.default_rng(20261207)
    seg_mb = 2
    nseg = chrom_mb // seg_mb
    dens = np.clip(np.exp(np.log(1500.0) + 0.9 * rng.standard_normal((n_chrom, nseg))), 25, 7500)
    chrom, pos = [], []
    for c in range(n_chrom):
        for k in range(nseg):
            cnt = int(round(dens[c, k] * seg_mb))
            lo = k * seg_mb * 1_000_000 + 1
            p = np.sort(rng.choice(np.arange(lo, lo + seg_mb * 1_000_000), size=cnt, replace=False))
            chrom += [str(c + 1)] * cnt
            pos.append(p)
    pos = np.concatenate(pos)
    m = pos.size
    fam = (25, 10, n - 250)
    rows, sub, _ = synth.make_bed_rows_chunked(4243, n, m, family=fam, keep_codes_every=50)
    samples = [f"S{i + 1:05d}" for i in range(n)]
    pre = os.path.join(d, "geno")
    with open(pre + ".fam", "w") as f:
        for s in samples:
            f.write(f"{s} {s} 0 0 0 -9\n")
    with open(pre + ".bim", "w") as f:
        f.write("".join(f"{chrom[i]}\trs{i + 1}\t0\t{int(pos[i])}\tA\tG\n" for i in range(m)))
    with open(pre + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(rows.tobytes())
    Y, _ = synth.polygenic_pheno(12, sub, genes)
    C = rng.standard_normal((n, n_cov))
    Y += 0.5 * C.sum(1, keepdims=True)
    ids, gc, st, en, sd, _ = synth.make_genes(6, genes, [str(c + 1) for c in range(n_chrom)],
                                              chrom_mb * 1_000_000, body=1)
    with open(os.path.join(d, "pheno.tsv"), "w") as f:  # 9 significant digits: the tables stay a few hundred MB
        f.write("sample\t" + "\t".join(ids) + "\n")
        for i, smp in enumerate(samples):
            f.write(smp + "\t" + "\t".join(f"{v:.9g}" for v in Y[i]) + "\n")
    synth.write_covar(os.path.join(d, "covar.tsv"), samples, C)
    synth.write_gff(os.path.join(d, "genes.gff"), ids, gc, st, en, sd)
    return m


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--genes", type=int, default=100)
    ap.add_argument("--perm", type=int, default=1000)
    ap.add_argument("--models", default="lmm,lm")
    ap.add_argument("--lognormal", action="store_true", help="lognormal cis-window sizes (see above)")
    ap.add_argument("--perm-rng", choices=("host", "device"), default="host",
                    help="host: the reference's seeded shuffles built on the host; device: permutations drawn "
                         "on the GPU (eqtl --perm-rng device)")
    ap.add_argument("--reference", type=int, nargs=2, metavar=("GENES", "PERM"),
                    help="also time the reference program (oracle/_ref/eqtl, all host threads) on GENES genes "
                         "of median window size with --perm PERM and extrapolate to the workload by the "
                         "window sizes and permutation count")
    args = ap.parse_args()
    exe = os.path.join(PKG, "bin", "eqtl")
    with tempfile.TemporaryDirectory(prefix="eqtl_perm_") as d:
        t_gen = time.perf_counter()
        m = make_case_lognormal(d, args.genes) if args.lognormal else make_case(d, args.genes)
        t_gen = time.perf_counter() - t_gen
        for model in args.models.split(","):
            cmd = [exe, "-b", os.path.join(d, "geno"), "-e", os.path.join(d, "pheno.tsv"), "-g",
                   os.path.join(d, "genes.gff"), "-c", os.path.join(d, "covar.tsv"), "--model", model, "--mode",
                   "cis", "-w", "1000000", "--perm", str(args.perm), "--perm-rng", args.perm_rng,
                   "-o", os.path.join(d, "out")]
            t0 = time.perf_counter()
            r = subprocess.run(cmd, capture_output=True, text=True, env={**os.environ, "EQTL_TRACE": "1"})
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                sys.exit(f"{model}: eqtl failed: {r.stderr[-2000:]}")
            stages = {"prep": 0.0, "scan": 0.0, "refine": 0.0}
            perm_cols = 0
            perm_ms = 0.0
            for ln in r.stderr.splitlines():
                mt = re.match(r"\[eqtl trace\] device stages of (\d+) columns \(ms\):(.*)", ln)
                if mt and int(mt.group(1)) != args.genes:  # the permutation scans
                    kv = mt.group(2).split()
                    for k, v in zip(kv[0::2], kv[1::2]):
                        if k in stages:
                            stages[k] += float(v)
                mt = re.match(r"\[eqtl trace\] permutations: device scan of (\d+) columns ([\d.]+) ms", ln)
                if mt:
                    perm_cols += int(mt.group(1))
                    perm_ms += float(mt.group(2))
            win = []
            with open(os.path.join(d, f"out.{model}.cis.region.tsv")) as f:
                next(f)
                for ln in f:
                    win.append(int(ln.split("\t")[3]))
            win = np.array(win)
            # host-side phases of the permutation driver (EQTL_TRACE): time since
            # the previous mark, summed over the batches
            host = {}
            kinds = (("columns ready", "wait for host-built columns"), ("drawn on the device", "device draws"),
                     ("device scan", "device scans"),
                     ("p_emp", "p_emp and beta fits"), ("setup", "setup"))
            for ln in r.stderr.splitlines():
                mt = re.match(r"\[eqtl trace\] permutations: (.*) ([\d.]+) ms$", ln)
                if mt:
                    for key, name in kinds:
                        if key in mt.group(1):
                            host[name] = host.get(name, 0.0) + float(mt.group(2))
            print(json.dumps({"workload": "cis permutations", "model": model, "perm_rng": args.perm_rng,
                              "n_samples": 1000, "n_snps": m,
                              "genes": args.genes, "perm": args.perm, "covariates": 15,
                              "window_snps_mean": float(win.mean()) if win.size else 0.0,
                              "window_snps_percentiles": {q: int(np.percentile(win, q)) for q in (0, 5, 50, 95, 100)}
                              if win.size else {},
                              "tests_observed": int(win.sum()), "generate_s": t_gen, "wall_s": wall,
                              "trace_ms": host,
                              "perm_columns": perm_cols, "perm_device_call_ms": perm_ms,
                              "perm_stage_ms": stages,
                              "perm_columns_per_s": perm_cols / (perm_ms / 1e3) if perm_ms else None}))
            if args.reference:
                print(json.dumps(reference_estimate(d, model, win, args.reference[0], args.reference[1],
                                                    args.perm)), flush=True)


def reference_estimate(d: str, model: str, win: np.ndarray, k: int, perm: int, perm_full: int) -> dict:
    """The reference program on the k genes whose windows are closest to the
    median, with --perm perm and without permutations; the difference per
    (window SNP, permutation) scaled by the workload's sum of window sizes
    and its permutation count."""
    exe = os.path.join(os.path.dirname(PKG), "oracle", "_ref", "eqtl")
    if not os.path.exists(exe):
        return {"reference": "oracle/_ref/eqtl not built"}
    with open(os.path.join(d, "pheno.tsv")) as f:
        head = f.readline().rstrip("\n").split("\t")
        rows = [ln.rstrip("\n").split("\t") for ln in f]
    # region rows follow the phenotype table's gene order (-t 1 below)
    pick = np.argsort(np.abs(win - np.median(win)), kind="stable")[:k]
    cols = [0] + [1 + int(i) for i in sorted(pick)]
    sub = os.path.join(d, "pheno_ref.tsv")
    with open(sub, "w") as f:
        f.write("\t".join(head[c] for c in cols) + "\n")
        for r in rows:
            f.write("\t".join(r[c] for c in cols) + "\n")
    threads = str(os.cpu_count() or 1)
    times = {}
    for b in (0, perm):
        cmd = [exe, "-b", os.path.join(d, "geno"), "-e", sub, "-g", os.path.join(d, "genes.gff"), "-c",
               os.path.join(d, "covar.tsv"), "--model", model, "--mode", "cis", "-w", "1000000", "--perm", str(b),
               "-t", threads, "-o", os.path.join(d, "ref")]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True)
        times[b] = time.perf_counter() - t0
        if r.returncode != 0:
            return {"reference": "failed: " + r.stderr[-500:]}
    snps = float(win[pick].sum())
    per = (times[perm] - times[0]) / (snps * perm)
    return {"reference": "oracle/_ref/eqtl", "model": model, "threads": int(threads), "genes": k, "perm": perm,
            "window_snps": snps, "wall_s_no_perm": times[0], "wall_s_perm": times[perm],
            "s_per_window_snp_perm": per, "estimate_s_full": per * float(win.sum()) * perm_full}


if __name__ == "__main__":
    main()
