"""GPU test of the allocation-free GRM entry point (eqtl_grm_noalloc) against
the regular path (eqtl_geno_load_bed + eqtl_grm) on the same genotypes.

Collected last (file name) so that it also runs after every other GPU test
has used the device; it passes alone as well."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _genotypes(seed, n_file, m, miss_rate=0.02):
    from eqtl_b200 import synth
    rng = np.random.default_rng(seed)
    af = rng.uniform(0.0, 0.5, size=m)
    af[::97] = 0.0                      # monomorphic rows: skipped by the GRM
    g = rng.binomial(2, af[:, None], size=(m, n_file)).astype(np.int8)
    g[rng.random((m, n_file)) < miss_rate] = -1
    g[::211, : n_file // 4] = -1         # heavily missing rows: dropped by max_miss
    return synth.pack_bed_rows(g)


@pytest.mark.parametrize("n_file,n,m", [(700, 450, 5000), (512, 512, 2048), (97, 61, 300)])
def test_grm_noalloc_matches_grm(n_file, n, m):
    import torch
    from eqtl_b200 import capi
    rows = _genotypes(n + m, n_file, m)
    rng = np.random.default_rng(n)
    cols = np.sort(rng.choice(n_file, size=n, replace=False)).astype(np.int32)
    kw = dict(miss_hand=capi.MISS_IMPUTE, max_miss=0.1, maf_min=0.01)
    with capi.Context(0) as c:
        c.load_bed(rows, n_file, cols, **kw)
        K_ref, N_ref, mu_ref = c.grm()
        bed_d = torch.from_numpy(rows).cuda()
        col_d = torch.from_numpy(cols).cuda()
        # outputs allocated up front, as a caller that cannot allocate has them
        outs = [(torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda"),
                 torch.full((n * (n + 1) // 2,), -1, dtype=torch.int32, device="cuda")) for _ in range(2)]
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for K_d, N_d in outs:  # two calls in a row: the scratch restarts from zero
            mu = c.grm_noalloc(bed_d.data_ptr(), m, rows.shape[1], col_d.data_ptr(), n, K_d.data_ptr(),
                               N_d.data_ptr(), **kw)
            torch.cuda.synchronize()
            # no device memory was taken by the call (the scratch array and the
            # kernels were set up when the context was opened)
            assert torch.cuda.mem_get_info()[0] == free0
            assert mu == mu_ref
            np.testing.assert_array_equal(N_d.cpu().numpy(), N_ref)
            # both paths accumulate FP32 tile partials (FP16 hi/lo operands)
            # into FP64, over different K ranges: agree to the GRM's own
            # tolerance against the FP64 oracle, twice over
            Kh = K_d.cpu().numpy()
            np.testing.assert_array_equal(Kh, Kh.T)
            np.testing.assert_allclose(Kh, K_ref, rtol=0, atol=4e-6 * np.abs(K_ref).max())


def test_grm_noalloc_rejects_oversize_n():
    import torch
    from eqtl_b200 import capi
    n = capi.GRM_NOALLOC_MAX_N + 1
    with capi.Context(0) as c:
        bed_d = torch.zeros((4, (n + 3) // 4), dtype=torch.uint8, device="cuda")
        col_d = torch.arange(n, dtype=torch.int32, device="cuda")
        K_d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        with pytest.raises(capi.EqtlError, match="static scratch limit"):
            c.grm_noalloc(bed_d.data_ptr(), 4, bed_d.shape[1], col_d.data_ptr(), n, K_d.data_ptr())
