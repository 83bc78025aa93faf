"""The eqtl host program (eqtl_b200/bin/eqtl) against outputs of the reference
program itself (tests/golden/): the same command lines, every pairs / top /
region file and the GCTA GRM files. Each command line runs twice: on the
golden PLINK files (-b) and on the same genotypes as a VCF (-v; the
reference's own VCF reader needs htslib, absent here, so the golden outputs
of the .bed runs are the reference for both).

Tolerances: LM pairs carry the FP64 refinement (log10 p within 1e-5, beta
within 1e-6 relative); LMM adds the REML optimiser difference (1e-4 and
1e-5). ACAT p uses the condition-aware bound of the parity tests (1e-3 plus
3 |dlog10 acat / dt| times the screening error of t, from the oracle).
Permutation p_emp is exact for the LM (same seeded shuffles, FP64 tests).
LMM permutations shuffle residuals in eigen-coordinates, so they depend on
the eigenvector signs, which differ between the reference's eigensolver
(Eigen) and cuSOLVER: runs with LMM permutations install the reference
eigensolver's basis of the run's GRM (ref_<tag>.basis.bin, made by
tests/golden/make_golden.py) through EQTL_LMM_BASIS, and then p_emp is
exact and p_beta / shapes within 5%, as for the LM.

The reference's own test panel (case "refdata", tests/golden/make_refdata.py)
runs from its converted .bed and from its original VCF."""
import json
import os
import subprocess

import numpy as np
import pytest

import driver
import restate as R
import refargs
import tsvcmp
from gpu_util import T_ERR

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIN = os.path.join(os.path.dirname(GOLD), "..", "eqtl_b200", "bin", "eqtl")


def _manifest(case):
    return json.load(open(os.path.join(GOLD, case, "manifest.json")))


def _runs():
    out = []
    for c in sorted(os.listdir(GOLD)):
        if not os.path.isdir(os.path.join(GOLD, c)):
            continue
        for tag, r in _manifest(c)["runs"].items():
            if r["argv"][0] != "fission":  # the fission subcommand has its own tests
                out.append((c, tag, r["argv"]))
    return out


def _skip_src(case, src):
    """Cases that carry their own VCF (the reference's test panel, "vcf" in
    the manifest) run from it ("vcf_orig") instead of from VCFs written here."""
    own = _manifest(case).get("vcf")
    if src == "vcf_orig" and not own:
        pytest.skip("no VCF of its own")
    if src in ("vcf", "vcf_ds") and own:
        pytest.skip("runs from the case's own VCF")


_SENS = {}


def _acat_sens(case, tag, argv, model, scope):
    """gene -> |d log10 acat_p / d t| of one model and scope, from the file
    made with the fixtures when there is one, else from the oracle."""
    key = (case, tag)
    if key not in _SENS:
        f = os.path.join(GOLD, case, f"ref_{tag}.sens.json")
        if os.path.exists(f):
            _SENS[key] = json.load(open(f))
        else:
            ora = driver.Scanner(refargs.options_from_argv(argv, os.path.join(GOLD, case)))
            ora.run()
            _SENS[key] = ora.sens_by
    return _SENS[key].get(f"{model}.{scope}", {})


def _basis_env(argv, case_dir, tag):
    """EQTL_LMM_BASIS for a run with LMM permutations (see the module text)."""
    env = dict(os.environ)
    env.pop("EQTL_LMM_BASIS", None)
    f = os.path.join(case_dir, f"ref_{tag}.basis.bin")
    if "--perm" in argv and os.path.exists(f):
        env["EQTL_LMM_BASIS"] = f
    return env


def bed_to_vcf(prefix: str, out_path: str, ds: bool = False) -> None:
    """The same genotypes as a gzip-compressed VCF: ALT = A1 (the counted
    allele), REF = A2, IDs and positions from the .bim. With `ds` every record
    also carries FORMAT/DS with the same dosages ("." where the call is
    missing), which the program then reads instead of GT. The index next to
    it (needed by cis scans) holds no sequences: records are read in file
    order."""
    from eqtl_b200 import synth
    rows, n_file, fam, bim = R.read_bed(prefix)
    i = np.arange(n_file)
    codes = (rows[:, i // 4] >> (2 * (i % 4))) & 3
    dosage = np.array([2, -1, 1, 0], np.int8)[codes]
    dsv = np.where(dosage < 0, np.nan, dosage.astype(np.float64)) if ds else None
    synth.write_vcf(out_path, fam, [b[0] for b in bim], [b[3] for b in bim], [b[1] for b in bim],
                    [b[5] for b in bim], [b[4] for b in bim], dosage, ds=dsv)
    synth.write_tabix_header(out_path)


def _run(argv, case_dir, out_prefix, src="bed", tmp=None, env=None):
    a = list(argv)
    a[a.index("-o") + 1] = out_prefix
    if src in ("vcf", "vcf_ds"):  # the same genotypes through -v (GT, or DS)
        vcf = os.path.join(str(tmp), "geno.vcf.gz" if src == "vcf" else "geno_ds.vcf.gz")
        if not os.path.exists(vcf):
            bed_to_vcf(os.path.join(case_dir, a[a.index("-b") + 1]), vcf, ds=src == "vcf_ds")
        k = a.index("-b")
        a[k:k + 2] = ["-v", vcf]
    elif src == "vcf_orig":  # the VCF the case's .bed was converted from
        k = a.index("-b")
        a[k:k + 2] = ["-v", json.load(open(os.path.join(case_dir, "manifest.json")))["vcf"]]
    r = subprocess.run([os.path.abspath(BIN)] + a, cwd=case_dir, capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.gpu
@pytest.mark.parametrize("src", ["bed", "vcf", "vcf_ds", "vcf_orig"])
@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" in r[2]])
def test_cli_make_grm(case, tag, argv, src, tmp_path):
    _skip_src(case, src)
    d = os.path.join(GOLD, case)
    out = str(tmp_path / "out")
    _run(argv, d, out, src, tmp_path)
    ref = os.path.join(d, f"ref_{tag}")
    assert open(out + ".grm.id").read() == open(ref + ".grm.id").read()
    N, Nr = (np.fromfile(p + ".grm.N.bin", dtype=np.float32) for p in (out, ref))
    assert np.array_equal(N, Nr)
    K, Kr = (np.fromfile(p + ".grm.bin", dtype=np.float32) for p in (out, ref))
    np.testing.assert_allclose(K, Kr, rtol=0, atol=2e-6 * np.abs(Kr).max())


@pytest.mark.gpu
@pytest.mark.parametrize("src", ["bed", "vcf", "vcf_ds", "vcf_orig"])
@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" not in r[2]])
def test_cli_scan_matches_reference(case, tag, argv, src, tmp_path):
    _skip_src(case, src)
    d = os.path.join(GOLD, case)
    out = str(tmp_path / "out")
    env = _basis_env(argv, d, tag)
    _run(argv, d, out, src, tmp_path, env)
    opt = refargs.options_from_argv(argv, d)
    scopes = ["gw"] if not opt.gff else {"cis": ["cis"], "trans": ["trans"], "gw": ["gw"],
                                         "all": ["cis", "trans"]}[opt.mode]
    errs = []
    for model in opt.out_models:
        tol = tsvcmp.Tol(log10p=1e-5, beta_rel=1e-6) if model == "lm" else tsvcmp.Tol(log10p=1e-4, beta_rel=1e-5)
        for scope in scopes:
            ref, got = os.path.join(d, f"ref_{tag}.{model}.{scope}"), f"{out}.{model}.{scope}"
            pthr = opt.pval_cis if scope == "cis" else opt.pval_trans
            for kind in ("pairs", "top"):
                hr, rr = tsvcmp.read_tsv(f"{ref}.{kind}.tsv")
                hg, gg = tsvcmp.read_tsv(f"{got}.{kind}.tsv")
                assert hr == hg
                errs += [f"{model}.{scope} {kind}: {e}" for e in tsvcmp.compare_pairs(rr, gg, tol, pthr)]
            hr, rr = tsvcmp.read_tsv(f"{ref}.region.tsv")
            hg, gg = tsvcmp.read_tsv(f"{got}.region.tsv")
            assert hr == hg
            if model == "lmm" and "--perm" in argv:
                assert "EQTL_LMM_BASIS" in env, "LMM permutation run without the reference's eigenbasis"
            errs += [f"{model}.{scope} region: {e}" for e in
                     tsvcmp.compare_region(rr, gg, tsvcmp.Tol(log10p=1e-3), check_perm=True,
                                           acat_sens=_acat_sens(case, tag, argv, model, scope), t_err=T_ERR)]
            # the gene order of each file is the reference's
            assert [r[0] for r in rr] == [g[0] for g in gg], (model, scope)
    assert not errs, "\n".join(errs[:40])


def test_cli_help_and_refusals():
    """Host-only behaviour of the command line (no GPU needed)."""
    exe = os.path.abspath(BIN)
    if not os.path.exists(exe):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--pval-cis" in r.stdout
    r = subprocess.run([exe, "-v", "x.vcf.gz", "-e", "p.tsv"], capture_output=True, text=True)
    assert r.returncode == 1 and "VCF" in r.stderr
    r = subprocess.run([exe, "-b", "geno"], capture_output=True, text=True)
    assert r.returncode == 1 and "missing -e/--pheno" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--model", "glmm"], capture_output=True, text=True)
    assert r.returncode == 1 and "glmm" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--model", "lm,glm", "--pheno-norm", "int"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "--pheno-norm int is incompatible with count model glm" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--maf", "0.7"], capture_output=True, text=True)
    assert r.returncode == 1 and "--maf must be in [0,0.5]" in r.stderr
