"""Array-level oracle scans for the C-ABI parity tests: the same per-pair
arithmetic as oracle/restate.py applied to in-memory genotype / phenotype
arrays (no files). Test infrastructure only."""
from __future__ import annotations

import numpy as np

import restate as R


def windows_mask(snp_chrom, snp_pos, gene_chrom, gene_lo, gene_hi):
    """[m, G] True where SNP s lies in gene g's window."""
    return ((snp_chrom[:, None] == gene_chrom[None, :]) & (gene_chrom[None, :] >= 0) &
            (snp_pos[:, None] >= gene_lo[None, :]) & (snp_pos[:, None] <= gene_hi[None, :]))


def trans_lm(G_dos, Y, X, pthr, excl=None):
    """SNP-outer LM over kept dosages G_dos [m, n]; Y [n, G]; X [n, p].
    Returns per-gene dict arrays + pairs list of (snp, gene, stats)."""
    m, n = G_dos.shape
    Gn = Y.shape[1]
    p = X.shape[1]
    preps = [R.prep_lm(Y[:, g], X) for g in range(Gn)]
    af, ok = R.subset_maf(G_dos)
    Xt_g = G_dos @ X
    g_s = G_dos - (Xt_g @ preps[0].XtX_inv.T) @ X.T
    gtg = np.einsum("ij,ij->i", g_s, g_s)
    Ys = np.stack([pp.y_s for pp in preps], 1)
    gty = g_s @ Ys
    st = R.lm_stats(gtg[:, None], gty, np.array([pp.yty for pp in preps])[None, :], n, p)
    use = ok[:, None] & (np.ones((m, Gn), bool) if excl is None else ~excl)
    return summarize(st, use, pthr, n - p - 1)


def summarize(st, use, pthr, df):
    m, Gn = st["p"].shape
    out = {"n_tested": use.sum(0), "acat_p": np.ones(Gn), "acat_sens": np.zeros(Gn),
           "best_snp": np.full(Gn, -1), "best_p": np.full(Gn, 2.0)}
    pairs = {}
    for g in range(Gn):
        u = use[:, g]
        acc = R.AcatAcc()
        acc.add_many(st["p"][u, g])
        acc.add_sensitivity(st["p"][u, g], st["stat"][u, g], df)
        out["acat_p"][g] = acc.p()
        out["acat_sens"][g] = acc.log10_sensitivity()
        idx = np.nonzero(u)[0]
        if idx.size:
            k = idx[np.argmin(st["p"][idx, g])]
            out["best_snp"][g] = k
            out["best_p"][g] = st["p"][k, g]
        for s in idx[st["p"][idx, g] <= pthr]:
            pairs[(int(s), g)] = {k2: float(st[k2][s, g]) for k2 in ("beta", "se", "stat", "p", "r2")}
    out["stats"] = st
    return out, pairs


def trans_lmm(G_dos, Y, X, Q, lam, pthr, excl=None, deltas=None):
    """SNP-outer LMM (src/scan_trans_lmm.cpp:82-251) over kept dosages;
    deltas[g] (optional, NaN = optimise) fixes gene g's REML delta."""
    m, n = G_dos.shape
    Gn = Y.shape[1]
    p = X.shape[1]
    fix = (lambda g: None) if deltas is None else (lambda g: None if np.isnan(deltas[g]) else float(deltas[g]))
    preps = [R.prep_lmm(Y[:, g], X, Q, lam, fix(g)) for g in range(Gn)]
    af, ok = R.subset_maf(G_dos)
    Gt = G_dos @ Q
    cols = [R.lmm_stats_gtil(pp, Gt) for pp in preps]
    st = {k: np.stack([c[k] for c in cols], 1) for k in cols[0]}
    use = ok[:, None] & (np.ones((m, Gn), bool) if excl is None else ~excl)
    out, pairs = summarize(st, use, pthr, n - p - 1)
    out["delta"] = np.array([pp.delta for pp in preps])
    return out, pairs


def glm(G_dos, Y, X, pthr, excl=None):
    """NB-GLM score test of every (SNP, gene) pair over kept dosages
    (prep_glm_nb / test_glm_nb, src/model_glm.cpp:74-132); a pair counts as
    tested when the subset gate passes and p is finite (a gene whose null fit
    failed tests nothing)."""
    m, n = G_dos.shape
    Gn = Y.shape[1]
    preps = [R.prep_glm_nb(Y[:, g], X) for g in range(Gn)]
    af, ok = R.subset_maf(G_dos)
    cols = [R.test_glm_nb_many(pp, G_dos) for pp in preps]
    st = {k: np.stack([c[k] for c in cols], 1) for k in cols[0]}
    use = ok[:, None] & np.isfinite(st["p"]) & (np.ones((m, Gn), bool) if excl is None else ~excl)
    out, pairs = summarize(st, use, pthr, None)
    out["phi"] = np.array([pp.phi for pp in preps])
    out["converged"] = np.array([pp.converged for pp in preps])
    return out, pairs
