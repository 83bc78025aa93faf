"""GPU parity: --pheno-norm int on the device (eqtl_pheno_int,
src/util.cpp:132-206) against the oracle's restatement, column by column:
continuous values, heavy ties (counts), both signs of zero, values that are
not finite (kept, and left out of the ranks), a column with one finite value
(unchanged), and a large column."""
import numpy as np
import pytest

import driver

pytestmark = pytest.mark.gpu


def test_pheno_int_matches_oracle():
    from eqtl_b200 import capi
    rng = np.random.default_rng(17)
    n = 777
    cols = [rng.standard_normal(n),
            rng.poisson(1.5, n).astype(np.float64),           # many ties
            np.where(rng.random(n) < 0.5, -0.0, 0.0) + rng.integers(0, 3, n),
            rng.standard_normal(n)]
    cols[3][rng.random(n) < 0.1] = np.nan
    cols[3][5] = np.inf
    one = np.full(n, np.nan)
    one[7] = 3.0
    cols.append(one)
    Y = np.column_stack(cols)
    with capi.Context(0) as c:
        got = c.pheno_int(Y)
        big = rng.gamma(2.0, 1.0, (20000, 3)).round(2)         # ties at 2 decimals, n > a block's worth
        got_big = c.pheno_int(big)
    for j in range(Y.shape[1]):
        ref = driver.inverse_normal_transform(Y[:, j])
        fin = np.isfinite(Y[:, j])
        assert np.array_equal(np.isfinite(got[:, j]), fin)
        np.testing.assert_array_equal(got[~fin, j], Y[~fin, j])
        np.testing.assert_allclose(got[fin, j], ref[fin], rtol=1e-13, atol=1e-15)
    for j in range(big.shape[1]):
        np.testing.assert_allclose(got_big[:, j], driver.inverse_normal_transform(big[:, j]), rtol=1e-13, atol=1e-15)
