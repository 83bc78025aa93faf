"""GPU parity of the fission subcommand: PEER on the device (eqtl_peer,
src/fission.cpp:104-275) against the oracle's restatement at FP64 tolerance
from the same starting values, over many iterations of a matrix with real
factor structure; and the command line's factors against the reference
program's golden files (six printed digits)."""
import json
import os
import subprocess

import numpy as np
import pytest

import restate as R

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "eqtl_b200", "bin", "eqtl")
CASE = os.path.join(ROOT, "tests", "golden", "fission")


def _read(path):
    rows = [ln.rstrip("\n").split("\t") for ln in open(path)]
    return [r[0] for r in rows[1:]], np.array([[float(v) for v in r[1:]] for r in rows[1:]])


def _structured(k):
    rng = np.random.default_rng(k)
    n, G = 150, 400
    Y = rng.standard_normal((n, 6)) @ rng.standard_normal((6, G)) * 2.0 + rng.standard_normal((n, G))
    Y[rng.random((n, G)) < 0.01] = np.nan
    return Y, rng.standard_normal((n, k)), rng.standard_normal((G, k))


@pytest.mark.parametrize("k,iters", [(4, 40), (12, 25)])
def test_peer_matches_oracle(k, iters):
    """The update rule drifts along nearly neutral directions (rotations of
    the factors that the ARD prior barely resists), so after tens of
    iterations it amplifies rounding: the oracle itself moves by d0 when Y
    moves by 1e-15 relative. The device must agree to 10 d0 there, and to
    1e-9 after 8 iterations, before any amplification."""
    from eqtl_b200 import capi
    Y, X0, W0 = _structured(k)
    Xr, itr = R.peer_factors(Y, k, iters, 1e-12, X0, W0)
    Yp = Y * (1 + 1e-15 * np.random.default_rng(99).standard_normal(Y.shape))
    d0 = np.abs(R.peer_factors(Yp, k, iters, 1e-12, X0, W0)[0] - Xr).max()
    X8r, _ = R.peer_factors(Y, k, 8, 1e-12, X0, W0)
    with capi.Context(0) as c:
        X, it = c.peer(Y, k, iters, 1e-12, X0, W0)
        X8, it8 = c.peer(Y, k, 8, 1e-12, X0, W0)
    assert it == itr and it8 == 8
    np.testing.assert_allclose(X8, X8r, rtol=1e-9, atol=1e-12 * np.abs(X8r).max())
    assert np.abs(X - Xr).max() <= 10 * d0 + 1e-12 * np.abs(Xr).max(), (np.abs(X - Xr).max(), d0)


@pytest.mark.parametrize("tag", ["counts", "cont", "covar"])
def test_fission_cli_matches_reference(tag, tmp_path):
    argv = json.load(open(os.path.join(CASE, "manifest.json")))["runs"][tag]["argv"]
    a = list(argv)
    a[a.index("-o") + 1] = str(tmp_path / "out")
    r = subprocess.run([BIN] + a, cwd=CASE, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    for part in ("Y1", "Y2"):
        assert open(tmp_path / f"out.{part}.tsv").read() == open(os.path.join(CASE, f"ref_{tag}.{part}.tsv")).read()
    s_got, F = _read(tmp_path / "out.factors.tsv")
    s_ref, Fr = _read(os.path.join(CASE, f"ref_{tag}.factors.tsv"))
    assert s_got == s_ref
    np.testing.assert_allclose(F, Fr, rtol=1e-5, atol=1e-5 * np.abs(Fr).max())
