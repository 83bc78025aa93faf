"""Generates the golden fixtures under tests/golden/<case>/.

Each case is a seeded synthetic PLINK data set (eqtl_b200.synth) plus the
outputs of the reference eqtl program itself, built from the reference's own
sources by `make -C oracle` (oracle/_ref/eqtl). Run from the repository root:

    make -C oracle REF=<reference tree> && python tests/golden/make_golden.py [case ...]

The fixtures are small (n=120 samples, 800 SNPs, 40 genes) so they commit
cheaply; larger parity cases are generated on the fly by the GPU tests.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from eqtl_b200 import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "eqtl")

# name -> (generator params, list of runs (tag, argv tail))
CASES = {
    "small": dict(
        geno=dict(seed=101, n=120, m=800, n_chrom=3, chrom_len=5_000_000, family=(4, 5, 100),
                  miss_rate=0.01, maf_lo=0.02),
        genes=dict(seed=102, n_genes=40, body=1000),
        pheno=dict(kind="lm", seed=103, n_cov=2),
        runs=[
            ("all", ["--model", "lm,lmm", "--mode", "all", "-w", "500000", "--pval-cis", "1e-2",
                     "--pval-trans", "1e-2", "-t", "2"]),
            ("gw", ["--model", "lm,lmm", "--mode", "gw", "--pval-trans", "1e-2", "-t", "1"]),
            ("perm", ["--model", "lm,lmm", "--mode", "all", "-w", "500000", "--pval-cis", "1e-2",
                      "--pval-trans", "1e-3", "--perm", "30", "--seed", "7", "--perm-trans-thr", "1e-2",
                      "--perm-trans-top", "5", "-t", "2"]),
            ("filter", ["--model", "lm", "--mode", "all", "-w", "500000", "--miss-hand", "filter",
                        "--maf", "0.1", "--pval-cis", "1e-2", "--pval-trans", "1e-2", "-t", "1"]),
            ("int", ["--model", "lm,lmm", "--mode", "trans", "--pheno-norm", "int", "--pval-trans",
                     "1e-2", "-t", "1"]),
            ("fast", ["--model", "lmm", "--mode", "all", "-w", "500000", "--pval-cis", "1e-2",
                      "--pval-trans", "1e-2", "--fast", "-t", "2"]),
            ("grm", ["--make-grm"]),
        ]),
    "counts": dict(
        geno=dict(seed=301, n=120, m=800, n_chrom=3, chrom_len=5_000_000, family=None,
                  miss_rate=0.01, maf_lo=0.02),
        genes=dict(seed=302, n_genes=30, body=1000),
        pheno=dict(kind="counts", seed=303, n_cov=2),
        runs=[
            ("all", ["--model", "glm", "--mode", "all", "-w", "500000", "--pval-cis", "1e-2",
                     "--pval-trans", "1e-2", "-t", "2"]),
            ("gw", ["--model", "glm", "--mode", "gw", "--pval-trans", "1e-2", "-t", "1"]),
            ("mixed", ["--model", "lm,glm", "--mode", "trans", "--miss-hand", "filter", "--maf", "0.05",
                       "--pval-trans", "5e-3", "-t", "1"]),
            ("perm", ["--model", "glm", "--mode", "all", "-w", "500000", "--pval-cis", "1e-2",
                      "--pval-trans", "1e-2", "--perm", "20", "--seed", "11", "-t", "1"]),
        ]),
    "nogff": dict(
        geno=dict(seed=201, n=96, m=600, n_chrom=2, chrom_len=3_000_000, family=None,
                  miss_rate=0.02, maf_lo=0.01),
        genes=dict(seed=202, n_genes=24, body=1),
        pheno=dict(kind="lmm", seed=203, n_cov=0),
        runs=[
            ("gw", ["--model", "lm,lmm", "--pval-trans", "5e-2", "--max-miss", "0.05", "-t", "1"]),
            ("grm", ["--make-grm", "--max-miss", "0.05"]),
        ]),
    # per-gene sample sets: some genes miss phenotype values (two of them at
    # the same samples, one with only 2 values left, so it drops out), and in
    # the *_cna runs one sample misses a covariate value, so no gene keeps
    # every analysis sample; cis_cna also takes the reference's per-thread
    # cis path (-t 2)
    "nakeep": dict(
        geno=dict(seed=501, n=110, m=700, n_chrom=3, chrom_len=5_000_000, family=(4, 5, 90),
                  miss_rate=0.01, maf_lo=0.02),
        genes=dict(seed=502, n_genes=30, body=1000),
        pheno=dict(kind="lm", seed=503, n_cov=2),
        na=dict(seed=504, genes=9, most=6, shared=(3, 4), sparse=11),
        cov_na=(17, 1),
        runs=[
            ("trans", ["--model", "lm,lmm", "--mode", "trans", "--pval-trans", "1e-2", "-t", "1"]),
            ("gw", ["--model", "lm,lmm", "--mode", "gw", "--pval-trans", "1e-2", "-t", "1"]),
            ("trans_cna", ["--model", "lm,lmm", "--mode", "trans", "--pval-trans", "1e-2", "-t", "1"]),
            ("cis", ["--model", "lm,lmm", "--mode", "cis", "-w", "500000", "--pval-cis", "1e-2", "-t", "1"]),
            ("cis_cna", ["--model", "lm,lmm", "--mode", "cis", "-w", "500000", "--pval-cis", "1e-2", "-t", "2"]),
            ("int", ["--model", "lm,lmm", "--mode", "trans", "--pheno-norm", "int", "--pval-trans", "1e-2",
                     "-t", "1"]),
        ]),
}


def plant_na(Y, na: dict):
    """NaN phenotype values: na["genes"] genes (from gene 1 on) miss 1 to
    na["most"] samples each; gene na["shared"][1] misses the same samples as
    gene na["shared"][0]; gene na["sparse"] keeps only 2 samples."""
    import numpy as np
    rng = np.random.default_rng(na["seed"])
    n, G = Y.shape
    Y = Y.copy()
    a, b = na["shared"]
    for g in range(1, 1 + na["genes"]):
        if g == b:
            continue
        Y[rng.choice(n, int(rng.integers(1, na["most"] + 1)), replace=False), g] = np.nan
    Y[:, b] = np.where(np.isnan(Y[:, a]), np.nan, Y[:, b])
    Y[2:, na["sparse"]] = np.nan
    return Y


def build_case(name: str, spec: dict) -> None:
    d = os.path.join(HERE, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    g = synth.make_genotypes(**spec["geno"])
    synth.write_plink(os.path.join(d, "geno"), g)
    gs = spec["genes"]
    chroms = sorted(set(g.chrom), key=g.chrom.index)
    ids, gc, st, en, sd, tss = synth.make_genes(gs["seed"], gs["n_genes"], chroms,
                                                spec["geno"]["chrom_len"], body=gs["body"])
    ph = spec["pheno"]
    if ph["kind"] == "counts":
        Y, C = synth.make_pheno_counts(ph["seed"], g, gs["n_genes"], ph["n_cov"], n_trans=10)
    elif ph["kind"] == "lm":
        Y, C = synth.make_pheno_lm(ph["seed"], g, gs["n_genes"], ph["n_cov"], cis_effects=True,
                                   gene_tss=tss, gene_chrom=gc, window=500_000, n_trans=10)
    else:
        Y, C, _ = synth.make_pheno_lmm(ph["seed"], g, gs["n_genes"], ph["n_cov"], n_trans=10)
    if "na" in spec:
        Y = plant_na(Y, spec["na"])
    synth.write_pheno(os.path.join(d, "pheno.tsv"), g.samples, ids, Y)
    have_cov = C.shape[1] > 0
    if have_cov:
        synth.write_covar(os.path.join(d, "covar.tsv"), g.samples, C)
    if "cov_na" in spec:
        Cn = C.copy()
        Cn[spec["cov_na"]] = float("nan")
        synth.write_covar(os.path.join(d, "covar_na.tsv"), g.samples, Cn)
    have_gff = name != "nogff"
    if have_gff:
        synth.write_gff(os.path.join(d, "genes.gff"), ids, gc, st, en, sd)
    manifest = {"runs": {}}
    for tag, argv in spec["runs"]:
        cmd = [REF, "-b", "geno"]
        if "--make-grm" not in argv:
            cmd += ["-e", "pheno.tsv"]
            if have_gff:
                cmd += ["-g", "genes.gff"]
            if have_cov:
                cmd += ["-c", "covar_na.tsv" if tag.endswith("_cna") else "covar.tsv"]
        cmd += argv + ["-o", f"ref_{tag}"]
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"{name}/{tag} failed: {r.stderr}")
        manifest["runs"][tag] = {"argv": cmd[1:]}
    for f in os.listdir(d):
        if ".tmp." in f:
            os.remove(os.path.join(d, f))
    with open(os.path.join(d, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


# -k: a GRM written by the reference's --make-grm for a wider sample set
# ("gwide": 12 more samples than the analysis fileset, in a shuffled order),
# then sliced by sample ID to the analysis samples. The phenotype table lists
# the samples in yet another order and holds 3 samples absent from the
# genotypes, so the analysis order differs from both the .fam and the
# .grm.id order.
KGRM_RUNS = [
    ("grmw", ["-b", "gwide", "--make-grm"]),
    ("k", ["-b", "geno", "--model", "lm,lmm", "--mode", "all", "-k", "ref_grmw", "-w", "500000", "--pval-cis",
           "1e-2", "--pval-trans", "1e-2", "-t", "2"]),
    ("kperm", ["-b", "geno", "--model", "lmm", "--mode", "all", "-k", "ref_grmw", "-w", "500000", "--pval-cis",
               "1e-2", "--pval-trans", "1e-3", "--perm", "30", "--seed", "5", "--perm-trans-thr", "1e-2",
               "--perm-trans-top", "5", "-t", "2"]),
]


def build_kgrm_case() -> None:
    import numpy as np
    d = os.path.join(HERE, "kgrm")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    n, n_wide = 120, 132
    g = synth.make_genotypes(401, n=n_wide, m=800, n_chrom=3, chrom_len=5_000_000, family=(4, 5, n_wide - 20),
                             miss_rate=0.01, maf_lo=0.02)
    rng = np.random.default_rng(402)
    perm = rng.permutation(n_wide)
    wide = synth.Genotypes(g.codes[:, perm], g.chrom, g.pos, g.ids, g.a1, g.a2, [g.samples[i] for i in perm], g.af)
    synth.write_plink(os.path.join(d, "gwide"), wide)
    sub = synth.Genotypes(g.codes[:, :n], g.chrom, g.pos, g.ids, g.a1, g.a2, g.samples[:n], g.af)
    synth.write_plink(os.path.join(d, "geno"), sub)
    chroms = sorted(set(g.chrom), key=g.chrom.index)
    ids, gc, st, en, sd, tss = synth.make_genes(403, 30, chroms, 5_000_000, body=1000)
    Y, C = synth.make_pheno_lm(404, sub, len(ids), 2, cis_effects=True, gene_tss=tss, gene_chrom=gc,
                               window=500_000, n_trans=8)
    extra = 3
    Yx = np.vstack([Y, rng.standard_normal((extra, Y.shape[1]))])
    Cx = np.vstack([C, rng.standard_normal((extra, C.shape[1]))])
    names = sub.samples + [f"X{i + 1:03d}" for i in range(extra)]
    order = rng.permutation(n + extra)
    synth.write_pheno(os.path.join(d, "pheno.tsv"), [names[i] for i in order], ids, Yx[order])
    synth.write_covar(os.path.join(d, "covar.tsv"), names, Cx)
    synth.write_gff(os.path.join(d, "genes.gff"), ids, gc, st, en, sd)
    manifest = {"runs": {}}
    for tag, argv in KGRM_RUNS:
        cmd = [REF] + argv[:2]
        if "--make-grm" not in argv:
            cmd += ["-e", "pheno.tsv", "-g", "genes.gff", "-c", "covar.tsv"]
        cmd += argv[2:] + ["-o", f"ref_{tag}"]
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"kgrm/{tag} failed: {r.stderr}")
        manifest["runs"][tag] = {"argv": cmd[1:]}
    for f in os.listdir(d):
        if ".tmp." in f:
            os.remove(os.path.join(d, f))
    with open(os.path.join(d, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


def write_bases(case_names=None) -> None:
    """For every golden run that has LMM permutations, the eigenbasis the
    reference's own eigensolver gives for that run's GRM (oracle/_ref/eigsolve
    on the oracle's FP64 GRM, or on the sliced -k file), written as
    ref_<tag>.basis.bin: n float64 eigenvalues, then the n x n eigenvectors
    column by column. LMM permutations shuffle residuals in eigen-
    coordinates, so with this basis installed a run reproduces the
    reference's permutation p-values exactly."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    import driver
    import refargs
    import restate as R
    for c in sorted(os.listdir(HERE)):
        cd = os.path.join(HERE, c)
        if not os.path.isdir(cd) or (case_names and c not in case_names):
            continue
        man = json.load(open(os.path.join(cd, "manifest.json")))
        for tag, r in man["runs"].items():
            argv = r["argv"]
            if argv[0] == "fission" or "--perm" not in argv:
                continue
            opt = refargs.options_from_argv(argv, cd)
            if "lmm" not in opt.out_models:
                continue
            K = driver.Scanner(opt).grm()
            Q, lam = R.make_lmm_basis(R.sparsify_grm(K, 1e-4) if opt.fast else K)
            with open(os.path.join(cd, f"ref_{tag}.basis.bin"), "wb") as f:
                f.write(np.ascontiguousarray(lam, dtype=np.float64).tobytes())
                f.write(np.asfortranarray(Q, dtype=np.float64).tobytes(order="F"))
            print("basis", c, tag, K.shape[0])


# The fission subcommand (data thinning + PEER factors) on phenotype tables
# only: counts (binomial thinning) and continuous values with a missing entry
# (Gaussian fission), with and without covariate residualisation.
FISSION_RUNS = [
    ("counts", ["-e", "counts.tsv", "--peer-factors", "4", "--epsilon", "0.4", "--seed", "7"]),
    ("cont", ["-e", "cont.tsv", "--peer-factors", "5", "--seed", "3", "--fission-tol", "1e-9",
              "--fission-max-iter", "300"]),
    ("covar", ["-e", "cont.tsv", "-c", "covar.tsv", "--peer-factors", "3", "--epsilon", "0.3"]),
]


def build_fission_case() -> None:
    import numpy as np
    d = os.path.join(HERE, "fission")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    rng = np.random.default_rng(5)
    n, G = 60, 80
    samples = [f"S{i:03d}" for i in range(n)]
    genes = [f"G{j:03d}" for j in range(G)]
    Yc, C = synth.make_pheno_counts(11, None, G, 2, n=n)
    Yg = rng.standard_normal((n, G)) + rng.standard_normal((n, 3)) @ rng.standard_normal((3, G))
    Yg[3, 7] = np.nan
    synth.write_pheno(os.path.join(d, "counts.tsv"), samples, genes, Yc)
    synth.write_pheno(os.path.join(d, "cont.tsv"), samples, genes, Yg)
    synth.write_covar(os.path.join(d, "covar.tsv"), samples[5:], C[5:])
    manifest = {"runs": {}}
    for tag, argv in FISSION_RUNS:
        cmd = [REF, "fission"] + argv + ["-o", f"ref_{tag}"]
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"fission/{tag} failed: {r.stderr}")
        manifest["runs"][tag] = {"argv": cmd[1:]}
    with open(os.path.join(d, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    if not os.path.exists(REF):
        raise SystemExit("build the reference first: make -C oracle REF=<reference tree>")
    only = sys.argv[1:]                      # case names to (re)build; all by default
    if only and only[0] == "--bases":        # only the LMM eigenbasis files of existing cases
        write_bases(only[1:])
        raise SystemExit(0)
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        build_case(name, spec)
        print("built", name)
    if not only or "kgrm" in only:
        build_kgrm_case()
        print("built kgrm")
    if not only or "fission" in only:
        build_fission_case()
        print("built fission")
    write_bases(only or None)
