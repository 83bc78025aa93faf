"""Refusals of the eqtl program's VCF input (-v) that happen before any
device work: -v together with -b, and BCF files. (The reading and the
filters, which parse the calls on the device, are in test_gpu_vcf.py.)"""
import os
import subprocess

import pytest


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "eqtl_b200", "bin", "eqtl")


def test_vcf_input_refusals(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    r = subprocess.run([BIN, "-v", "a.vcf.gz", "-b", "geno", "-e", "p.tsv"], capture_output=True, text=True)
    assert r.returncode == 1 and "use only one of -v/--vcf or -b/--bfile" in r.stderr
    bcf = tmp_path / "x.bcf"
    bcf.write_bytes(b"BCF\x02\x02rest\n")
    ph = tmp_path / "p.tsv"
    ph.write_text("sample\tG1\nS1\t0.1\n")
    r = subprocess.run([BIN, "-v", str(bcf), "-e", str(ph)], capture_output=True, text=True)
    assert r.returncode == 1 and "BCF input" in r.stderr