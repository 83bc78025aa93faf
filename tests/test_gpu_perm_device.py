"""Device-drawn permutations (eqtl_pheno_permute, --perm-rng device).

1. The columns the device builds equal the CPU restatement of the mode
   (oracle/philox.py: Philox4x32-10 keys, stable order, LM and LMM forms)
   bit for bit, for several shapes including n not a multiple of 4.
2. A scan of the resident columns equals a scan of the same columns passed
   from the host.
3. The host program's p_emp with device draws agrees with its p_emp with the
   reference's seeded shuffles (host draws, exact against the reference
   program) within Monte-Carlo error at 1,000 permutations, for LM and LMM,
   cis and trans stage 2; device draws are reproducible and depend on the
   seed.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import tsvcmp

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import philox  # noqa: E402

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIN = os.path.join(os.path.dirname(GOLD), "..", "eqtl_b200", "bin", "eqtl")


@pytest.fixture(scope="module")
def ctx():
    from eqtl_b200 import capi
    with capi.Context(0) as c:
        yield c


@pytest.mark.parametrize("n,G,B,seed", [(2, 1, 3, 1), (37, 5, 17, 42), (120, 7, 64, 2**40 + 9), (1001, 3, 5, 7)])
@pytest.mark.parametrize("form", ["lm", "lmm"])
def test_device_columns_match_restatement(ctx, n, G, B, seed, form):
    rng = np.random.default_rng(n + G)
    base = rng.normal(size=(n, G))
    X = np.column_stack([np.ones(n), rng.normal(size=n)])
    keys = np.array([philox.fnv1a64(f"GENE{g:05d}") for g in range(G)], np.uint64)
    xb0 = dinv = None
    if form == "lmm":
        xb0 = rng.normal(size=(n, G))
        dinv = rng.uniform(0.05, 3.0, size=(n, G))
        dinv[0, 0] = 0.0  # clamped at 1e-12 like the host build
    got = ctx.pheno_permute(base, X, keys, B, seed, xb0, dinv, out=True)
    want = philox.permuted_columns(base, [int(k) for k in keys], B, seed, xb0, dinv)
    np.testing.assert_array_equal(got, want)


def test_resident_scan_equals_host_columns(ctx):
    from eqtl_b200 import synth
    n, m, G, B = 160, 900, 6, 25
    g = synth.make_genotypes(4, n=n, m=m, n_chrom=2, chrom_len=2_000_000, miss_rate=0.01, maf_lo=0.02)
    Y, C = synth.make_pheno_lm(5, g, G, 2, cis_effects=False, n_trans=10, beta_sd=0.4)
    X = np.column_stack([np.ones(n), C])
    ctx.load_bed(synth.pack_bed_rows(g.codes), n, np.arange(n))
    resid = Y - X @ np.linalg.lstsq(X, Y, rcond=None)[0]
    keys = [philox.fnv1a64(f"g{j}") for j in range(G)]
    cols = ctx.pheno_permute(resid, X, keys, B, 11, out=True)
    g_res, p_res, _ = ctx.scan_trans_lm(None, None, pthr=1e-2)
    g_host, p_host, _ = ctx.scan_trans_lm(cols, X, pthr=1e-2)
    assert np.array_equal(g_res, g_host)
    assert np.array_equal(p_res, p_host)


def _run(argv, out):
    a = list(argv)
    a[a.index("-o") + 1] = out
    r = subprocess.run([os.path.abspath(BIN)] + a, cwd=os.path.join(GOLD, "small"), capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]


def _p_emp(prefix, model, scope):
    h, rows = tsvcmp.read_tsv(f"{prefix}.{model}.{scope}.region.tsv")
    i = h.index("p_emp")
    return {r[0]: float(r[i]) for r in rows if r[i] not in ("NA", "nan")}


def test_cli_device_draws_agree_with_host_draws(tmp_path):
    import json
    argv = json.load(open(os.path.join(GOLD, "small", "manifest.json")))["runs"]["perm"]["argv"]
    B = 1000
    argv = list(argv)
    argv[argv.index("--perm") + 1] = str(B)
    host, dev, dev2, dev3 = (str(tmp_path / t) for t in ("host", "dev", "dev2", "dev3"))
    _run(argv, host)
    _run(argv + ["--perm-rng", "device"], dev)
    _run(argv + ["--perm-rng", "device"], dev2)
    k = argv.index("--seed")
    _run(argv[:k] + ["--seed", "8"] + argv[k + 2:] + ["--perm-rng", "device"], dev3)
    z, compared, differ = [], 0, 0
    for model in ("lm", "lmm"):
        for scope in ("cis", "trans"):
            ph, pd = _p_emp(host, model, scope), _p_emp(dev, model, scope)
            assert set(ph) == set(pd), (model, scope)
            assert pd == _p_emp(dev2, model, scope)  # reproducible
            p3 = _p_emp(dev3, model, scope)
            differ += sum(p3[g] != pd[g] for g in pd)
            for gname in ph:
                a, b = ph[gname], pd[gname]
                pbar = min(max(0.5 * (a + b), 1.0 / (B + 1)), 1 - 1.0 / (B + 1))
                sd = np.sqrt(2 * pbar * (1 - pbar) / B)
                assert abs(a - b) <= 5 * sd + 2.0 / (B + 1), (model, scope, gname, a, b)
                z.append((a - b) / sd)
                compared += 1
    assert compared >= 20, compared
    assert abs(float(np.mean(z))) <= 4.0 / np.sqrt(len(z)), np.mean(z)
    assert differ > 0  # another seed draws other permutations
