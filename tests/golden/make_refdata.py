"""Builds tests/golden/refdata/ from the reference's own test panel
(data/test of WWz33/eqtl: 200 samples, 11,760 biallelic SNPs on one contig,
1,000 genes, one covariate, GT-only VCF) and the outputs of the reference
program on it.

The reference reads VCF through htslib, which this image lacks, so its runs
here read the same genotypes converted to PLINK .bed, with A1 = ALT (the
counted allele) and A2 = REF, IDs and positions from the VCF. A diploid GT
call counts its ALT alleles; a call with a missing allele is missing, as the
reference's VcfSession::parse_record does (src/vcf_session.cpp:220-258). The
GPU tests then run the host program on both the .bed and the original VCF
and compare every output file with the reference's.

    make -C oracle REF=<reference tree> && python tests/golden/make_refdata.py [path/to/reference]

The reference tree defaults to $EQTL_REFERENCE, else /root/reference.
"""
from __future__ import annotations

import gzip
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from eqtl_b200 import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "eqtl")
OUT = os.path.join(HERE, "refdata")

# cfg1's settings on the panel (cis LM and LMM at 1e-5 with the default 1 Mb
# window), a looser cis threshold on a narrower window (the panel has no cis
# signal at 1e-5), the trans scope, and LM gene-level permutations.
RUNS = [
    ("cis", ["--model", "lm,lmm", "--mode", "cis", "--pval-cis", "1e-5", "-t", "8"]),
    ("cisw", ["--model", "lm,lmm", "--mode", "cis", "-w", "250000", "--pval-cis", "1e-3", "-t", "8"]),
    ("trans", ["--model", "lm,lmm", "--mode", "trans", "--pval-trans", "1e-5", "-t", "8"]),
    ("perm", ["--model", "lm", "--mode", "cis", "--pval-cis", "1e-5", "--perm", "20", "--seed", "3", "-t", "8"]),
]


def vcf_to_bed(vcf: str, prefix: str) -> int:
    samples, chrom, pos, ids, ref, alt, rows = None, [], [], [], [], [], []
    with gzip.open(vcf, "rt") as f:
        for ln in f:
            if ln.startswith("##"):
                continue
            t = ln.rstrip("\n").split("\t")
            if ln.startswith("#CHROM"):
                samples = t[9:]
                continue
            if "," in t[4]:
                raise SystemExit("multi-allelic record in the panel")
            fmt = t[8].split(":")
            gi = fmt.index("GT")
            d = np.empty(len(samples), np.int8)
            for j, call in enumerate(t[9:]):
                gt = call.split(":")[gi].replace("|", "/").split("/")
                if len(gt) != 2 or "." in gt:
                    d[j] = -1
                else:
                    d[j] = int(gt[0]) + int(gt[1])
            chrom.append(t[0])
            pos.append(int(t[1]))
            ids.append(t[2])
            ref.append(t[3])
            alt.append(t[4])
            rows.append(d)
    codes = np.array(rows)
    g = synth.Genotypes(codes, chrom, np.array(pos, np.int64), ids, alt, ref, samples, np.zeros(len(rows)))
    synth.write_plink(prefix, g)
    return len(rows)


def write_sensitivities(manifest) -> None:
    """Per run, model and scope, each gene's |d log10 acat_p / d t| from the
    oracle (the ACAT tolerance of the GPU tests), as ref_<tag>.sens.json, so
    the GPU tests need not rerun the oracle on the 1,000 genes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import driver
    import refargs
    for tag, r in manifest["runs"].items():
        sc = driver.Scanner(refargs.options_from_argv(r["argv"], OUT))
        sc.run()
        with open(os.path.join(OUT, f"ref_{tag}.sens.json"), "w") as f:
            json.dump({k: {g: round(v, 6) for g, v in d.items()} for k, d in sc.sens_by.items()}, f, indent=0,
                      sort_keys=True)


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "data", "test")
    if not os.path.exists(REF):
        raise SystemExit("build the reference first: make -C oracle REF=<reference tree>")
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    os.makedirs(OUT)
    for a, b in (("test.vcf.gz", "test.vcf.gz"), ("test.vcf.gz.tbi", "test.vcf.gz.tbi"),
                 ("test.pheno.tsv", "pheno.tsv"), ("test.covar.tsv", "covar.tsv"), ("test.gff", "genes.gff")):
        shutil.copyfile(os.path.join(src, a), os.path.join(OUT, b))
    m = vcf_to_bed(os.path.join(OUT, "test.vcf.gz"), os.path.join(OUT, "geno"))
    manifest = {"vcf": "test.vcf.gz", "runs": {}}
    for tag, argv in RUNS:
        cmd = [REF, "-b", "geno", "-e", "pheno.tsv", "-g", "genes.gff", "-c", "covar.tsv"] + argv + \
              ["-o", f"ref_{tag}"]
        r = subprocess.run(cmd, cwd=OUT, capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"refdata/{tag} failed: {r.stderr}")
        manifest["runs"][tag] = {"argv": cmd[1:]}
    for f in os.listdir(OUT):
        if ".tmp." in f:
            os.remove(os.path.join(OUT, f))
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    write_sensitivities(manifest)
    print(f"refdata: {m} records, {len(RUNS)} runs")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EQTL_REFERENCE", "/root/reference"))
