"""GPU unit test of the device Student-t tail (the epilogue's table
interpolation) against the reference's p_from_t (src/util.cpp:247-262)
restated in oracle/restate.py, on a dense (t, df) grid."""
import numpy as np
import pytest

import restate as R

pytestmark = pytest.mark.gpu

DEFER_NL = 14.0  # pairs with -log10 p above this take the FP64 host path


def _grid():
    return np.concatenate([[0.0, 1e-9, 1e-6, 1e-3, 0.5, 0.99, 1.0, 1.01], np.linspace(-8, 8, 4001),
                           np.geomspace(8, 1e4, 400), np.geomspace(1e4, 1e21, 60)]).astype(np.float32)


@pytest.mark.parametrize("df", [1.0, 5.0, 30.0, 118.0, 295.0, 997.0, 1998.0])
@pytest.mark.parametrize("smem", [False, True])
def test_t_tail_matches_p_from_t(df, smem):
    from eqtl_b200 import capi
    t = _grid()
    with capi.Context(0) as c:
        nl, term, fl = c.t_tail(df, t, use_smem=smem)
    p = R.p_from_t(t.astype(np.float64), df)
    want_nl = -np.log10(np.maximum(p, 1e-300))
    deferred = (fl & 2) != 0
    used = (fl & 1) != 0
    # -log10 p to FP32 accuracy (relative 2e-6; 1e-8 absolute covers the
    # reference's own ~1e-11 error near p = 1)
    ok = ~deferred
    np.testing.assert_allclose(nl[ok], want_nl[ok], rtol=2e-6, atol=1e-8)
    # deferral: every pair past -log10 p = 14 goes to the host, and every
    # pair near t = 0 where the reference's x = df / (df + t^2) is quantised;
    # no pair in between
    at = np.abs(t.astype(np.float64))
    tiny = (at > 0) & (at < 3e-6)
    mid = (at > 1e-3) & (want_nl < DEFER_NL * (1 - 1e-5))
    assert np.all(deferred[(want_nl > DEFER_NL * (1 + 1e-5)) | tiny])
    assert not np.any(deferred[mid | (at == 0)])
    # ACAT entry on the device: p < 1 - 1e-12 (AcatAcc::add,
    # src/stats_extra.cpp:16-22) for pairs that are not deferred
    np.testing.assert_array_equal(used, (p < 1 - 1e-12) & ~deferred)
    # ACAT term tan((1/2 - p) pi) = +-cot(pi m), m = min(p, 1 - p): invert the
    # device term to m and compare in m, where FP32 precision is relative
    q = used & ~deferred
    m_ref = np.minimum(p[q], 1.0 - p[q])
    tq = term[q]
    assert np.all(((tq > 0) == (p[q] < 0.5)) | (np.abs(p[q] - 0.5) < 1e-6))
    m_dev = np.arctan2(1.0, np.abs(tq)) / np.pi  # = atan(1/|t|); m = 1/2 at a zero term
    rtol = 3e-6 * np.maximum(1.0, -np.log(m_ref))
    assert np.all(np.abs(m_dev - m_ref) <= rtol * m_ref + 2e-11), np.max(np.abs(m_dev - m_ref) / m_ref)
    # unused and deferred pairs contribute nothing on the device
    assert np.all(term[~q] == 0.0)


@pytest.mark.parametrize("df", [1.0, 5.0, 30.0, 118.0, 295.0, 997.0, 1998.0])
@pytest.mark.parametrize("smem", [False, True])
def test_acat_screen_matches_p_from_t(df, smem):
    """The scan epilogues' ACAT screen: the term from one table lookup,
    deferral by |t| (p <= 1e-14, and |t| near 0), the best-SNP score |t|."""
    from eqtl_b200 import capi
    t = _grid()
    with capi.Context(0) as c:
        key, term, fl = c.t_tail(df, t, use_smem=smem, screen=True)
    p = R.p_from_t(t.astype(np.float64), df)
    want_nl = -np.log10(np.maximum(p, 1e-300))
    at = np.abs(t.astype(np.float64))
    np.testing.assert_array_equal(key, np.abs(t))
    deferred = (fl & 2) != 0
    used = (fl & 1) != 0
    tiny = (at > 0) & (at < 3e-6)
    mid = (at > 1e-3) & (want_nl < DEFER_NL * (1 - 1e-3))
    assert np.all(deferred[(want_nl > DEFER_NL * (1 + 1e-3)) | tiny])
    assert not np.any(deferred[mid | (at == 0)])
    assert np.array_equal((fl & 4) != 0, deferred & (at < 1e-3))
    np.testing.assert_array_equal(used, (p < 1 - 1e-12) & ~deferred)
    q = used
    m_ref = np.minimum(p[q], 1.0 - p[q])
    tq = term[q]
    assert np.all(((tq > 0) == (p[q] < 0.5)) | (np.abs(p[q] - 0.5) < 1e-6))
    m_dev = np.arctan2(1.0, np.abs(tq)) / np.pi  # = atan(1/|t|); m = 1/2 at a zero term
    rtol = 3e-6 * np.maximum(1.0, -np.log(m_ref))
    assert np.all(np.abs(m_dev - m_ref) <= rtol * m_ref + 2e-11), np.max(np.abs(m_dev - m_ref) / m_ref)
    assert np.all(term[~q] == 0.0)
