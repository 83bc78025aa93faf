"""VCF input (-v) of the eqtl program, read on the host and parsed on the
device (BGZF members inflated on all host threads, the calls by
eqtl_vcf_parse), against the oracle's restatement of the reference's
VcfSession (src/vcf_session.cpp:148-305).

The cases cover the rules where VCF input differs from a .bed: multi-allelic
and ALT "." records are skipped; on X / Y / MT (with or without "chr") and for
haploid calls every call carries one allele, so the frequency that the
monomorphic test and --maf see is sum / ploidy, not mean / 2; filters run
over the analysis samples (the phenotype samples, in their own order); a
header that defines DS switches to FORMAT/DS dosages; plain, gzip and BGZF
files give the same GRM; DS values outside the device parser's exact fast
path are parsed on the host."""
import os
import re
import subprocess

import numpy as np
import pytest

import restate as R

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "eqtl_b200", "bin", "eqtl")


def _case(tmp):
    from eqtl_b200 import synth
    rng = np.random.default_rng(11)
    n = 60
    samples = [f"S{i:03d}" for i in range(n)]
    order = rng.permutation(n)[:50]  # analysis samples: 50 phenotype samples, shuffled
    chrom, pos, dos, hap = [], [], [], []

    def add(c, d, h=None):
        chrom.append(c)
        pos.append(1000 * (len(pos) + 1))
        dos.append(np.asarray(d, np.int8))
        hap.append(np.zeros(n, bool) if h is None else np.asarray(h, bool))

    for _ in range(30):  # diploid autosomes with 3% missing
        d = rng.binomial(2, rng.uniform(0.05, 0.5), n)
        d[rng.random(n) < 0.03] = -1
        add("1", d)
    add("1", np.zeros(n))                           # monomorphic
    d = rng.binomial(2, 0.3, n)
    d[:12] = -1                                     # 20% missing: above --max-miss 0.1
    add("1", d)
    males = np.arange(n) < 30
    for _ in range(8):  # X: haploid males, diploid females
        d = np.where(males, rng.binomial(1, 0.3, n), rng.binomial(2, 0.3, n))
        add("X", d, males)
    add("X", np.where(males, 1, 2), males)          # all ALT: af = 1 (mean / 2 would give 0.75)
    d = np.zeros(n)
    d[order[:4]] = 1
    add("Y", d, np.ones(n, bool))                   # af = 4/50 passes --maf 0.05 (mean / 2 would not)
    add("chrX", rng.binomial(1, 0.4, n), np.ones(n, bool))
    d = rng.binomial(2, 0.2, n)
    d[:5] = np.minimum(d[:5], 1)
    add("2", d, np.arange(n) < 5)                   # haploid calls on an autosome
    m = len(chrom)
    ids = [f"rs{i}" for i in range(m)]
    vcf = os.path.join(str(tmp), "g.vcf.gz")
    synth.write_vcf(vcf, samples, chrom, pos, ids, ["A"] * m, ["G"] * m, np.stack(dos), np.stack(hap), phased=True)
    # records that are not biallelic: appended as text
    import gzip
    with gzip.open(vcf, "at") as f:
        f.write("1\t99000\tm1\tA\tC,T\t.\tPASS\t.\tGT\t" + "\t".join(["0/1"] * n) + "\n")
        f.write("1\t99100\tm2\tA\t.\t.\tPASS\t.\tGT\t" + "\t".join(["0/0"] * n) + "\n")
    ph = os.path.join(str(tmp), "p.tsv")
    with open(ph, "w") as f:
        f.write("sample\tG1\n")
        for i in order:
            f.write(f"{samples[i]}\t{rng.standard_normal():.6f}\n")
    return vcf, ph, order


def test_vcf_reader_and_filters_match_restatement(tmp_path):
    vcf, ph, order = _case(tmp_path)
    r = subprocess.run([BIN, "-v", vcf, "-e", ph, "--make-grm", "--maf", "0.05", "--max-miss", "0.1", "-o",
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=300)
    err = r.stderr
    samples, recs, n_multi = R.read_vcf_gt(vcf)
    keep = R.vcf_keep(recs, order, 0.1, False, 0.05)
    m = re.search(r"VCF multi-allelic sites skipped \(biallelic only\): (\d+)", err)
    assert m and int(m.group(1)) == n_multi == 2, err[-2000:]
    m = re.search(r"VCF: (\d+) biallelic records of (\d+) on (\d+) samples", err)
    assert m and int(m.group(1)) == len(recs) and int(m.group(3)) == len(samples), err[-2000:]
    m = re.search(r"VCF: (\d+) of (\d+) biallelic records pass the filters on (\d+) samples", err)
    assert m, err[-2000:]
    assert (int(m.group(1)), int(m.group(2)), int(m.group(3))) == (int(keep.sum()), len(recs), 50)
    # the rules that differ from a .bed decide some records here
    chroms = [rc[0] for rc in recs]
    assert not keep[chroms.index("X") + 8]              # all-ALT X record
    assert keep[chroms.index("Y")]                      # rare Y record passes --maf on sum / ploidy
    assert r.returncode == 0, err[-2000:]





def _ds_case(tmp):
    """A VCF whose header declares FORMAT/DS: most records carry GT:DS with
    imputed dosages (some "." and one sample column cut short), two records
    carry GT only, one X record carries DS (ploidy 1 for every call)."""
    from eqtl_b200 import synth
    rng = np.random.default_rng(12)
    n = 40
    samples = [f"S{i:03d}" for i in range(n)]
    order = rng.permutation(n)[:32]
    m = 24
    chrom = ["1"] * (m - 3) + ["X", "2", "2"]
    pos = [1000 * (r + 1) for r in range(m)]
    gt = rng.binomial(2, 0.3, (m, n)).astype(np.int8)
    ds = np.clip(gt + rng.normal(0, 0.2, (m, n)), 0, 2)
    ds[rng.random((m, n)) < 0.05] = np.nan
    ds[3] = 0.0                                  # monomorphic in DS (GT would not be)
    ds[3, 0] = 0.0
    ds[5, :] = np.where(np.arange(n) % 2 == 0, np.nan, ds[5])   # half missing: above --max-miss
    ds[6] = 1e-4 * rng.random(n)                 # af below --maf
    ds[m - 3] = rng.uniform(0.995, 1.0, n)       # X: af = sum / calls > 0.99 (mean / 2 would be ~0.5)
    ds_rows = np.ones(m, bool)
    ds_rows[[1, m - 1]] = False                  # GT-only records
    ids = [f"rs{i}" for i in range(m)]
    vcf = os.path.join(str(tmp), "d.vcf.gz")
    synth.write_vcf(vcf, samples, chrom, pos, ids, ["A"] * m, ["G"] * m, gt, ds=ds, ds_rows=ds_rows)
    import gzip
    with gzip.open(vcf, "at") as f:             # a sample column without its DS subfield
        f.write("1\t99000\tcut\tA\tC\t.\tPASS\t.\tGT:DS\t" + "\t".join(["0/1"] + ["0/1:0.9"] * (n - 1)) + "\n")
    ph = os.path.join(str(tmp), "p.tsv")
    with open(ph, "w") as f:
        f.write("sample\tG1\n")
        for i in order:
            f.write(f"{samples[i]}\t{rng.standard_normal():.6f}\n")
    return vcf, ph, order


def test_vcf_ds_reader_and_filters_match_restatement(tmp_path):
    vcf, ph, order = _ds_case(tmp_path)
    r = subprocess.run([BIN, "-v", vcf, "-e", ph, "--make-grm", "--maf", "0.01", "--max-miss", "0.3", "-o",
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=300)
    err = r.stderr
    assert "FORMAT/DS present" in err and "using FORMAT/DS dosages" in err, err[-2000:]
    samples, recs, n_multi = R.read_vcf_dosage(vcf)
    assert sum(rc[7] for rc in recs) == len(recs) - 2
    keep = R.vcf_keep(recs, order, 0.3, False, 0.01)
    m = re.search(r"VCF: (\d+) of (\d+) biallelic records pass the filters on (\d+) samples", err)
    assert m, err[-2000:]
    assert (int(m.group(1)), int(m.group(2)), int(m.group(3))) == (int(keep.sum()), len(recs), 32)
    assert not keep[3] and not keep[5] and not keep[6]
    assert not keep[len(recs) - 4]               # the X record: af = sum / calls fails --maf 0.01
    assert keep.sum() >= len(recs) - 6
    assert np.isnan(recs[-1][5][0]) and recs[-1][5][1] == np.float32(0.9)
    assert r.returncode == 0, err[-2000:]


def test_vcf_cis_needs_index(tmp_path):
    from eqtl_b200 import synth
    vcf, ph, _ = _ds_case(tmp_path)
    gff = tmp_path / "g.gff"
    gff.write_text("##gff-version 3\n1\tsynth\tgene\t5000\t6000\t.\t+\t.\tID=G1;Name=G1\n")
    argv = [BIN, "-v", vcf, "-e", ph, "-g", str(gff), "--mode", "cis", "-o", str(tmp_path / "o")]
    r = subprocess.run(argv, capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "cis mode requires an indexed genotype file" in r.stderr, r.stderr[-2000:]
    synth.write_tabix_header(vcf)
    r = subprocess.run(argv, capture_output=True, text=True, timeout=300)
    assert "cis mode requires an indexed genotype file" not in r.stderr
    assert r.returncode == 0, r.stderr[-2000:]


def _grm_files(prefix):
    N = np.fromfile(prefix + ".grm.N.bin", dtype=np.float32)
    K = np.fromfile(prefix + ".grm.bin", dtype=np.float32)
    return K, N


@pytest.mark.parametrize("kind", ["ds_long", "gt"])
def test_vcf_containers_and_host_fallback(kind, tmp_path):
    """The same genotypes as plain text, one gzip member, BGZF and BCF2 give
    the same GRM, equal to the oracle's from its own reading of the file. With
    DS written to 17 significant digits every value misses the device's fast
    path and is parsed on the host."""
    from eqtl_b200 import synth
    rng = np.random.default_rng(7)
    n, m = 90, 700
    samples = [f"S{i:03d}" for i in range(n)]
    order = rng.permutation(n)[:80]
    gt = rng.binomial(2, rng.uniform(0.05, 0.5, m)[:, None], (m, n)).astype(np.int8)
    gt[rng.random((m, n)) < 0.02] = -1
    ds = None
    if kind == "ds_long":
        ds = np.clip(gt + rng.normal(0, 0.1, (m, n)), 0, 2)
        ds[gt < 0] = np.nan
    chrom = ["1"] * (m // 2) + ["2"] * (m - m // 2)
    pos = list(range(1, m + 1))
    ph = str(tmp_path / "p.tsv")
    with open(ph, "w") as f:
        f.write("sample\tG1\n")
        for i in order:
            f.write(f"{samples[i]}\t{rng.standard_normal():.6f}\n")
    outs = []
    for name, bgzf in (("g.vcf", False), ("g.vcf.gz", False), ("b.vcf.gz", True), ("g.bcf", True)):
        path = str(tmp_path / name)
        if name.endswith(".bcf"):
            synth.write_bcf(path, samples, chrom, pos, [f"rs{i}" for i in range(m)], ["A"] * m, ["G"] * m, gt, ds=ds)
        else:
            synth.write_vcf(path, samples, chrom, pos, [f"rs{i}" for i in range(m)], ["A"] * m, ["G"] * m, gt, ds=ds,
                            bgzf=bgzf, ds_text=(lambda v: "." if not np.isfinite(v) else "%.17g" % v)
                            if ds is not None else None)
        out = str(tmp_path / ("o_" + name.replace(".", "_")))
        r = subprocess.run([BIN, "-v", path, "-e", ph, "--make-grm", "--maf", "0.01", "-o", out], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(_grm_files(out))
    for K, N in outs[1:]:
        assert np.array_equal(N, outs[0][1]) and np.array_equal(K, outs[0][0])
    _, recs, _ = R.read_vcf_dosage(str(tmp_path / "g.vcf"))
    keep = R.vcf_keep(recs, order, 0.8, False, 0.01)
    rows = np.stack([rc[5] for rc, k in zip(recs, keep) if k]).astype(np.float32)
    dec = R.decode_dosage_rows(rows, order, "impute", 1.0, 0.0)
    Kr, Nr, _ = R.compute_grm(dec.dosage[dec.keep], dec.codes[dec.keep] < 0)
    K, N = outs[0]
    np.testing.assert_array_equal(N, Nr.astype(np.float32))
    np.testing.assert_allclose(K, R.grm_lower_f32(Kr), rtol=0, atol=2e-6 * np.abs(Kr).max())
