"""The eqtl program's VCF input (-v) where no device work is involved: the
refusals (-v together with -b, a BCF of another major version) and BCF2
files, whose typed binary calls are decoded on the host (the text VCF's
calls are parsed on the device: test_gpu_vcf.py). A BCF written from the
same genotypes as a VCF must give the records and filter decisions of the
oracle's reading of that VCF (src/vcf_session.cpp:148-305)."""
import os
import re
import subprocess

import numpy as np
import pytest

import restate as R


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "eqtl_b200", "bin", "eqtl")


def test_vcf_input_refusals(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    r = subprocess.run([BIN, "-v", "a.vcf.gz", "-b", "geno", "-e", "p.tsv"], capture_output=True, text=True)
    assert r.returncode == 1 and "use only one of -v/--vcf or -b/--bfile" in r.stderr
    bcf = tmp_path / "x.bcf"
    bcf.write_bytes(b"BCF\x01\x02rest\n")
    ph = tmp_path / "p.tsv"
    ph.write_text("sample\tG1\nS1\t0.1\n")
    r = subprocess.run([BIN, "-v", str(bcf), "-e", str(ph)], capture_output=True, text=True)
    assert r.returncode == 1 and "BCF input of an unsupported version" in r.stderr

@pytest.mark.parametrize("with_ds", [False, True])
def test_bcf_reader_and_filters_match_restatement(with_ds, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    from eqtl_b200 import synth
    rng = np.random.default_rng(4)
    n, m = 60, 400
    samples = [f"S{i:03d}" for i in range(n)]
    order = rng.permutation(n)[:50]
    gt = rng.binomial(2, rng.uniform(0.01, 0.5, m)[:, None], (m, n)).astype(np.int8)
    gt[rng.random((m, n)) < 0.03] = -1
    hap = np.zeros((m, n), bool)
    chrom = ["1"] * (m - 60) + ["X"] * 40 + ["2"] * 20
    males = np.arange(n) < 30
    hap[m - 60:m - 20] = males                     # X: haploid males
    hap[m - 20:, :4] = True                        # haploid calls on an autosome
    gt[hap] = np.minimum(gt[hap], 1)
    ds = None
    if with_ds:
        ds = np.clip(gt + rng.normal(0, 0.1, (m, n)), 0, 2).astype(np.float32)
        ds[gt < 0] = np.nan
    args = (samples, chrom, list(range(1, m + 1)), [f"rs{i}" for i in range(m)], ["A"] * m, ["G"] * m, gt, hap)
    vcf, bcf = str(tmp_path / "g.vcf"), str(tmp_path / "g.bcf")
    synth.write_vcf(vcf, *args, ds=ds)
    synth.write_bcf(bcf, *args, ds=ds)
    ph = str(tmp_path / "p.tsv")
    with open(ph, "w") as f:
        f.write("sample\tG1\n")
        for i in order:
            f.write(f"{samples[i]}\t{rng.standard_normal():.6f}\n")
    r = subprocess.run([BIN, "-v", bcf, "-e", ph, "--make-grm", "--maf", "0.05", "--max-miss", "0.1", "-o",
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=300)
    _, recs, _ = R.read_vcf_dosage(vcf)
    keep = R.vcf_keep(recs, order, 0.1, False, 0.05)
    m_ = re.search(r"VCF: (\d+) of (\d+) biallelic records pass the filters on (\d+) samples", r.stderr)
    assert m_, r.stderr[-2000:]
    assert (int(m_.group(1)), int(m_.group(2)), int(m_.group(3))) == (int(keep.sum()), len(recs), 50)
    assert ("using FORMAT/DS dosages" in r.stderr) == with_ds
    assert r.returncode == 0 or "no usable B200" in r.stderr, r.stderr[-2000:]
