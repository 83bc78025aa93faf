"""The fission subcommand's thinning on the host (eqtl fission, with the
standard library's distributions drawn in the reference's order,
src/fission.cpp:31-83,277-300): Y1 and Y2 are the reference program's,
byte for byte, for counts, continuous values with a missing entry, and a
covariate sample subset. The program writes them before it opens the GPU,
so this runs without one. Also the subcommand's refusals."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "eqtl_b200", "bin", "eqtl")
CASE = os.path.join(ROOT, "tests", "golden", "fission")


def _runs():
    man = json.load(open(os.path.join(CASE, "manifest.json")))
    return [(tag, r["argv"]) for tag, r in man["runs"].items()]


@pytest.mark.parametrize("tag,argv", _runs())
def test_fission_thinning_matches_reference(tag, argv, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    a = list(argv)
    a[a.index("-o") + 1] = str(tmp_path / "out")
    r = subprocess.run([BIN] + a, cwd=CASE, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 or "no usable B200" in r.stderr, r.stderr[-2000:]
    for part in ("Y1", "Y2"):
        got = open(tmp_path / f"out.{part}.tsv").read()
        ref = open(os.path.join(CASE, f"ref_{tag}.{part}.tsv")).read()
        assert got == ref, (tag, part)


def test_fission_refusals(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    r = subprocess.run([BIN, "fission", "--peer-factors", "3"], capture_output=True, text=True)
    assert r.returncode == 1 and "fission requires -e/--pheno" in r.stderr
    r = subprocess.run([BIN, "fission", "-e", "counts.tsv", "--epsilon", "1.5"], cwd=CASE, capture_output=True,
                       text=True)
    assert r.returncode == 1 and "--epsilon must be in (0,1)" in r.stderr
    r = subprocess.run([BIN, "fission", "-e", "counts.tsv", "--peer-factors", "80", "-o", str(tmp_path / "o")],
                       cwd=CASE, capture_output=True, text=True)
    assert r.returncode == 1 and "--peer-factors must be < min(n_samples, n_genes)" in r.stderr
