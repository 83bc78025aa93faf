"""CPU restatement of the reference scan orchestration (numpy).

TEST INFRASTRUCTURE ONLY (the checker; never imported by the product).
Restates src/scan.cpp:50-312 (run_eqtl_geno) for PLINK input and the LM/LMM
models: scope selection, per-gene complete-case preparation, SNP-outer
trans/gw scans, gene-outer cis scans, gene-level permutations, ACAT, BH, and
the pairs/top/region rows. Rows are returned as lists of tuples of the
printed fields; formatting follows src/output.cpp:8-110.
"""
from __future__ import annotations

import math
import os
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import restate as R  # noqa: E402


# ---------------------------------------------------------------------------
# Inputs  (src/pheno.cpp:17-196, src/annot.cpp:26-71, src/util.cpp:68-87)
# ---------------------------------------------------------------------------
def _split_line(line: str) -> List[str]:
    return line.split("\t") if "\t" in line else line.split()


def load_pheno(path: str):
    with open(path) as f:
        lines = f.read().splitlines()
    head = lines[0].strip()
    if head.startswith("#"):
        head = head[1:]
    header = _split_line(head)
    genes = [h.strip() for h in header[1:]]
    ids, rows = [], []
    for ln in lines[1:]:
        ln = ln.strip()
        if not ln or ln.startswith("#"):
            continue
        t = _split_line(ln)
        if len(t) != len(header):
            raise ValueError("pheno row column mismatch")
        ids.append(t[0].strip())
        rows.append([float("nan") if v in ("NA", "NaN", ".") else float(v) for v in t[1:]])
    seen, keep = {}, []
    for i, s in enumerate(ids):
        if s in seen:
            continue
        seen[s] = i
        keep.append(i)
    Y = np.array([rows[i] for i in keep], dtype=np.float64)
    return [ids[i] for i in keep], genes, Y


def load_covar(path: Optional[str], samples: List[str]) -> np.ndarray:
    n = len(samples)
    if not path:
        return np.ones((n, 1))
    ids, rows, first = [], [], True
    for ln in open(path):
        ln = ln.strip()
        if not ln or ln.startswith("#"):
            continue
        t = _split_line(ln)
        if len(t) < 2:
            continue
        if first:
            first = False

            def is_num(s):
                try:
                    float(s)
                    return True
                except ValueError:
                    return False
            if not is_num(t[1]):
                continue
        ids.append(t[0])
        rows.append([float(v) for v in t[1:]])
    m = {}
    for i, s in enumerate(ids):
        m.setdefault(s, i)
    raw = np.array([rows[m[s]] for s in samples], dtype=np.float64)
    has_int = any(np.all(np.abs(raw[:, j] - 1.0) <= 1e-12) for j in range(raw.shape[1]))
    return raw if has_int else np.column_stack([np.ones(n), raw])


def chrom_key(c: str) -> str:
    s = c
    if len(s) >= 3 and s[:3].lower() == "chr":
        s = s[3:]
    i = 0
    while i + 1 < len(s) and s[i] == "0":
        i += 1
    return s[i:]


def chrom_equal(a: str, b: str) -> bool:
    return a == b or chrom_key(a) == chrom_key(b)


@dataclass
class GeneLoc:
    chrom: str
    start: int
    end: int
    tss: int


def load_gff(path: str, id_key: str = "") -> Dict[str, GeneLoc]:
    out, multi = {}, set()
    for ln in open(path):
        if not ln or ln.startswith("#"):
            continue
        c = ln.rstrip("\n").split("\t")
        if len(c) < 9 or c[2] != "gene":
            continue
        attrs = {}
        for kv in c[8].strip().split(";"):
            kv = kv.strip()
            if "=" not in kv:
                continue
            k, v = kv.split("=", 1)
            attrs.setdefault(k.strip(), [x.strip() for x in v.split(",")])
        if id_key:
            gid = (attrs.get(id_key) or [""])[0]
        else:
            gid = (attrs.get("ID") or [""])[0] or (attrs.get("Name") or [""])[0] or \
                (attrs.get("gene_id") or [""])[0]
        if not gid:
            continue
        if gid.startswith("gene:"):
            gid = gid[5:]
        strand = c[6] if c[6] in ("+", "-") else "+"
        start, end = int(c[3]), int(c[4])
        if gid in out or gid in multi:
            if gid in out:
                del out[gid]
                multi.add(gid)
            continue
        out[gid] = GeneLoc(c[0], start, end, end if strand == "-" else start)
    return out


def inverse_normal_transform(y: np.ndarray) -> np.ndarray:
    """src/util.cpp:132-206 (Acklam + one Halley step; average ranks)."""
    y = y.copy()
    fin = np.isfinite(y)
    vals = y[fin]
    nf = vals.size
    if nf <= 1:
        return y
    order = np.argsort(vals, kind="stable")
    ranks = np.empty(nf)
    i = 0
    sv = vals[order]
    while i < nf:
        j = i + 1
        while j < nf and sv[j] == sv[i]:
            j += 1
        ranks[order[i:j]] = 0.5 * (i + 1 + j)
        i = j
    a = [-39.6968302866538, 220.9460984245205, -275.9285104469687, 138.3577518678900,
         -30.6647980661472, 2.506628277459239]
    b = [-54.4760987982241, 161.5858368580409, -155.6989798598867, 66.8013118877197,
         -13.28068155278571]
    c = [-0.007784894002430293, -0.3223964580411364, -2.4007582771618388, -2.5497325393437340,
         4.3746641414649678, 2.9381639826987831]
    d = [0.0077846957090414622, 0.32246712907003983, 2.4451341371429960, 3.7544086619074161]

    def qn(p):
        p = min(max(p, 1e-15), 1.0 - 1e-15)
        tgt = p
        neg = p > 0.5
        if neg:
            p = 1.0 - p
        if p < 0.02425:
            q = math.sqrt(-2.0 * math.log(p))
            v = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) / \
                ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0)
        else:
            q = p - 0.5
            r = q * q
            v = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q / \
                (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0)
        if neg:
            v = -v
        cdf = 0.5 * math.erfc(-v / math.sqrt(2.0))
        phi = math.exp(-0.5 * v * v) / math.sqrt(2.0 * math.pi)
        if phi > 1e-300:
            f = cdf - tgt
            den = 2.0 * phi * phi + f * v * phi
            if den != 0.0:
                v -= 2.0 * f * phi / den
        return v

    y[fin] = np.array([qn((r - 0.5) / nf) for r in ranks])
    return y


# ---------------------------------------------------------------------------
# Scan
# ---------------------------------------------------------------------------
@dataclass
class Options:
    bfile: str
    pheno: str
    out_models: tuple = ("lmm",)
    mode: str = "all"
    gff: str = ""
    covar: str = ""
    grm: str = ""
    window: int = 1_000_000
    pval_cis: float = 1e-5
    pval_trans: float = 1e-5
    miss_hand: str = "impute"
    max_miss: float = 0.8
    maf: float = 0.0
    perm: int = 0
    perm_trans_thr: float = 1e-5
    perm_trans_top: int = 1000
    seed: int = -1
    disable_beta_approx: bool = False
    pheno_norm: str = "none"
    threads: int = 1
    fast: bool = False


def fmt(v) -> str:
    return "%.10g" % v


@dataclass
class Summary:
    gene: str
    chrom: str = ""
    tss: int = 0
    n_tested: int = 0
    n_sig: int = 0
    acat: float = 1.0
    p_emp: float = float("nan")
    p_beta: float = float("nan")
    s1: float = 0.0
    s2: float = 0.0
    q: float = float("nan")
    acat_sens: float = 0.0   # |d log10 acat_p / d t| (see AcatAcc.log10_sensitivity)


def per_thread_written(rows, work_of_row, threads, n_works):
    """The rows of a pairs or top file as the reference's per-thread cis
    driver leaves them (src/scan_cis.cpp:29-160): thread t scans the works
    [t c, (t + 1) c), c = ceil(n_works / threads), into a temporary file, and
    the files are appended in thread order with `dst << in.rdbuf()`.
    Appending an empty file sets the stream's failbit, so nothing of that or
    any later thread reaches the output."""
    T = max(1, threads)
    c = -(-n_works // T) if n_works else 1
    has = [False] * T
    for w in work_of_row:
        has[w // c] = True
    ok, written = True, []
    for t in range(T):
        written.append(ok and has[t])
        ok = ok and has[t]
    return [r for r, w in zip(rows, work_of_row) if written[w // c]]


def pair_row(gene, snp_meta, h, n, loc, scope):
    chrom, pos, sid, ref, alt = snp_meta
    tss = fmt(float(pos - loc.tss)) if loc is not None else "NA"
    return (gene, sid, chrom, str(pos), ref, alt, fmt(h["af"]), fmt(h["beta"]), fmt(h["se"]),
            fmt(h["stat"]), fmt(h["p"]), fmt(h["r2"]), str(n), tss, scope)


def region_row(s: Summary):
    na = lambda v: "NA" if not math.isfinite(v) else fmt(v)
    return (s.gene, s.chrom, str(s.tss), str(s.n_tested), str(s.n_sig), fmt(s.acat), na(s.q),
            na(s.p_emp), na(s.p_beta), fmt(s.s1), fmt(s.s2))


def _hit(stats, i, af, j=None):
    ix = i if j is None else (i, j)
    return {"beta": stats["beta"][ix], "se": stats["se"][ix], "stat": stats["stat"][ix],
            "p": stats["p"][ix], "r2": stats["r2"][ix], "af": af}


class Scanner:
    def __init__(self, opt: Options):
        self.opt = opt
        samples_ph, self.genes, Y = load_pheno(opt.pheno)
        rows, n_file, fam, self.bim = R.read_bed(opt.bfile)
        famset = set(fam)
        order = [s for s in samples_ph if s in famset]
        pos_ph = {s: i for i, s in enumerate(samples_ph)}
        self.Y = Y[[pos_ph[s] for s in order]]
        fam_pos = {s: i for i, s in enumerate(fam)}
        self.samples = order
        self.X = load_covar(opt.covar, order)
        dec = R.decode_bed_rows(rows, n_file, [fam_pos[s] for s in order], opt.miss_hand,
                                opt.max_miss, opt.maf)
        self.dec = dec
        self.kept = np.nonzero(dec.keep)[0]
        self.annot = load_gff(opt.gff) if opt.gff else {}
        self.K = None

    # -- GRM ---------------------------------------------------------------
    def grm(self):
        if self.K is None:
            if self.opt.grm:
                self.K = load_grm_sliced(self.opt.grm, self.samples)
            else:
                k = self.kept
                self.K, _, _ = R.compute_grm(self.dec.dosage[k], self.dec.codes[k] < 0)
        return self.K

    def snp_meta(self, s):
        c, i, _, p, a1, a2 = self.bim[s]
        return (c, p, i, a2, a1)

    def gene_y(self, gi):
        y = self.Y[:, gi].copy()
        if self.opt.pheno_norm == "int":
            y = inverse_normal_transform(y)
        return y

    def build_ready(self, y, need_k):
        keep = np.nonzero(np.isfinite(y) & np.all(np.isfinite(self.X), axis=1))[0]
        if keep.size < 3:
            return None
        yk = y[keep]
        if np.max(np.abs(yk)) < 1e-15:
            return None
        K = self.grm()[np.ix_(keep, keep)] if need_k else None
        return keep, yk, self.X[keep], K

    def scopes(self):
        if not self.opt.gff:
            return ["gw"]
        return {"cis": ["cis"], "trans": ["trans"], "gw": ["gw"], "all": ["cis", "trans"]}[self.opt.mode]

    def in_cis(self, s, loc):
        c, _, _, p, _, _ = self.bim[s]
        if not chrom_equal(c, loc.chrom):
            return False
        lo = max(loc.start - self.opt.window, 1)
        return lo <= p <= loc.end + self.opt.window

    def run(self):
        res = {}
        self.sens_by = {}  # "model.scope" -> gene -> |d log10 acat_p / d t|
        for model in self.opt.out_models:
            for scope in self.scopes():
                before = dict(getattr(self, "sens", {}))
                self.sens = {}
                res[(model, scope)] = self.run_scope(model, scope)
                self.sens_by[f"{model}.{scope}"] = dict(self.sens)
                before.update(self.sens)
                self.sens = before
        return res

    # -- SNP-outer trans/gw (src/scan_trans_lm.cpp:41-163, src/scan_trans_lmm.cpp:82-251) --
    def run_scope(self, model, scope):
        opt = self.opt
        pthr = opt.pval_cis if scope == "cis" else opt.pval_trans
        if model == "glm":
            return self.run_glm(scope, pthr)
        if scope == "cis":
            return self.run_cis(model, pthr)
        jobs = []
        for gi, gene in enumerate(self.genes):
            loc = self.annot.get(gene) if opt.gff else None
            if opt.gff and loc is None and scope != "gw":
                continue
            if scope == "trans" and loc is None:
                continue
            ready = self.build_ready(self.gene_y(gi), need_k=False)
            if ready is None:
                continue
            jobs.append((gene, loc, ready))
        pairs, tops, summ = [], [], []
        if not jobs:
            return pairs, tops, []
        # genes whose keep sets differ run per keep set (the reference's
        # per-job paths, src/scan_trans_lm.cpp:121-151,
        # src/scan_trans_lmm.cpp:192-228): the SNP gate, residualisation and
        # (LMM) basis of each set's samples; pairs keep their (SNP, gene) order
        groups = {}
        for jg, job in enumerate(jobs):
            groups.setdefault(tuple(int(i) for i in job[2][0]), []).append(jg)
        summ = [None] * len(jobs)
        tops_by = [[] for _ in jobs]
        for keep_t, idxs in groups.items():
            keep0 = np.array(keep_t, dtype=np.int64)
            gjobs = [jobs[jg] for jg in idxs]
            X = gjobs[0][2][2]
            n, p = X.shape
            G = self.dec.dosage[self.kept][:, keep0]
            af_sub, ok = R.subset_maf(G)
            snps = self.kept[ok]
            G = G[ok]
            af_sub = af_sub[ok]
            ng = len(gjobs)
            if model == "lm":
                preps = [R.prep_lm(j[2][1], j[2][2]) for j in gjobs]
                Xt_g = G @ X
                g_s = G - (Xt_g @ preps[0].XtX_inv.T) @ X.T
                gtg = np.einsum("ij,ij->i", g_s, g_s)
                Ys = np.stack([pp.y_s for pp in preps], 1)
                gty = g_s @ Ys                                  # [m, G]
                st = R.lm_stats(gtg[:, None], gty, np.array([pp.yty for pp in preps])[None, :], n, p)
                degenerate = gtg < 1e-12
            else:
                K = self.grm()[np.ix_(keep0, keep0)]
                Q, lam = R.make_lmm_basis(R.sparsify_grm(K, 1e-4) if opt.fast else K)
                preps = [R.prep_lmm(j[2][1], j[2][2], Q, lam) for j in gjobs]
                Gt = G @ Q
                cols = [R.lmm_stats_gtil(pp, Gt) for pp in preps]
                st = {k: np.stack([c[k] for c in cols], 1) for k in cols[0]}
                degenerate = np.zeros(G.shape[0], dtype=bool)
            excl = np.zeros((len(snps), ng), dtype=bool)
            if scope == "trans":
                for j, (gene, loc, _) in enumerate(gjobs):
                    excl[:, j] = [self.in_cis(s, loc) for s in snps]
            topk = opt.perm_trans_top if opt.perm > 0 else 0
            for j, (gene, loc, ready) in enumerate(gjobs):
                s = Summary(gene)
                gtops = []
                if loc is not None:
                    s.chrom, s.tss = loc.chrom, loc.tss
                acc = R.AcatAcc()
                best_p, best = 2.0, None
                pv = st["p"][:, j]
                use = ~excl[:, j]
                s.n_tested = int(use.sum())
                acc.add_many(pv[use])
                acc.add_sensitivity(pv[use], st["stat"][:, j][use], n - p - 1)
                sig = use & (pv <= pthr)
                s.n_sig = int(sig.sum())
                for i in np.nonzero(sig)[0]:
                    pairs.append((int(snps[i]), idxs[j], pair_row(gene, self.snp_meta(snps[i]),
                                                             _hit(st, i, af_sub[i], j) if not degenerate[i]
                                                             else _p1(af_sub[i]), n, loc, scope)))
                cand = np.nonzero(use)[0]
                if cand.size:
                    k = cand[np.argmin(pv[cand])]   # first index on ties (strict <)
                    best_p, best = pv[k], k
                s.acat = acc.p()
                s.acat_sens = acc.log10_sensitivity()
                if best is not None and best_p <= pthr and best_p <= 1.0:
                    gtops.append(pair_row(gene, self.snp_meta(snps[best]),
                                         _hit(st, best, af_sub[best], j) if not degenerate[best]
                                         else _p1(af_sub[best]), n, loc, scope))
                if topk > 0 and best is not None and best_p < opt.perm_trans_thr and s.n_tested > 0:
                    cidx = np.nonzero(use & np.isfinite(pv) & (pv < opt.perm_trans_thr) & ~degenerate)[0]
                    cidx = cidx[np.argsort(pv[cidx], kind="stable")][:topk]
                    cached = [G[i] for i in cidx]
                    if cached:
                        self.perm(model, s, gene, ready, cached, best_p, preps[j], lmm_basis=(
                            (Q, lam) if model == "lmm" else None))
                summ[idxs[j]] = s
                tops_by[idxs[j]] = gtops
        for t in tops_by:
            tops.extend(t)
        pairs.sort(key=lambda t: (t[0], t[1]))
        return [p_[2] for p_ in pairs], tops, self.finish(summ)

    def finish(self, summ):
        q = R.bh_adjust([s.acat for s in summ])
        for s, qq in zip(summ, q):
            s.q = qq
        self.sens = getattr(self, "sens", {})
        self.sens.update({s.gene: s.acat_sens for s in summ})
        return [region_row(s) for s in summ]

    # -- cis (include/eqtl/scan_cis.hpp:15-185, src/scan_cis.cpp:18-163) ----
    def run_cis(self, model, pthr):
        opt = self.opt
        works = [(gi, g, self.annot[g]) for gi, g in enumerate(self.genes) if g in self.annot]
        if opt.threads > 1:
            works.sort(key=lambda w: (w[2].chrom, w[2].tss))
        basis = None
        if model == "lmm":
            K = self.grm()
            if K.shape[0] == len(self.samples):
                basis = R.make_lmm_basis(R.sparsify_grm(K, 1e-4) if opt.fast else K)
        pairs, tops, summ = [], [], []
        pair_w, top_w = [], []  # position in `works` of each pair's / top's gene
        bim_chrom = [b[0] for b in self.bim]
        for wi, (gi, gene, loc) in enumerate(works):
            y = self.gene_y(gi)
            if basis is not None and np.all(np.isfinite(y)) and np.all(np.isfinite(self.X)):
                keep, yk, Xk = np.arange(len(y)), y, self.X
                Q, lam = basis
            else:
                ready = self.build_ready(y, need_k=(model == "lmm"))
                if ready is None:
                    continue
                keep, yk, Xk, Kk = ready
                if model == "lmm":
                    Q, lam = R.make_lmm_basis(R.sparsify_grm(Kk, 1e-4) if opt.fast else Kk)
            lo = max(loc.start - opt.window, 1)
            hi = loc.end + opt.window
            win = [s for s in self.kept
                   if chrom_equal(bim_chrom[s], loc.chrom) and lo <= self.bim[s][3] <= hi]
            s = Summary(gene, loc.chrom, loc.tss)
            prep = R.prep_lm(yk, Xk) if model == "lm" else R.prep_lmm(yk, Xk, Q, lam)
            acc = R.AcatAcc()
            best_p, best_row = 2.0, None
            cached = []
            if win:
                G = self.dec.dosage[np.array(win)][:, keep]
                af_sub, ok = R.subset_maf(G)
                st = R.test_lm_many(prep, G) if model == "lm" else R.test_lmm_many(prep, G)
                n = len(keep)
                for i, snp in enumerate(win):
                    if not ok[i]:
                        continue
                    pv = st["p"][i]
                    s.n_tested += 1
                    acc.add_many([pv])
                    acc.add_sensitivity([pv], [st["stat"][i]], n - Xk.shape[1] - 1)
                    row = pair_row(gene, self.snp_meta(snp), _hit(st, i, af_sub[i]), n, loc, "cis")
                    if pv <= pthr:
                        pairs.append(row)
                        pair_w.append(wi)
                        s.n_sig += 1
                    if pv < best_p:
                        best_p, best_row = pv, row
                    if opt.perm > 0:
                        cached.append(G[i])
            s.acat = acc.p()
            s.acat_sens = acc.log10_sensitivity()
            if opt.perm > 0 and s.n_tested > 0:
                self.perm(model, s, gene, (keep, yk, Xk, None), cached, best_p, prep,
                          lmm_basis=(Q, lam) if model == "lmm" else None)
            if best_row is not None and best_p <= pthr and best_p <= 1.0:
                tops.append(best_row)
                top_w.append(wi)
            summ.append(s)
        if opt.threads > 1:
            pairs = per_thread_written(pairs, pair_w, opt.threads, len(works))
            tops = per_thread_written(tops, top_w, opt.threads, len(works))
        return pairs, tops, self.finish(summ)

    # -- NB GLM, gene-outer for every scope (src/scan.cpp:227-300 and, for cis
    # with -t > 1, src/scan_cis.cpp:18-115; per gene include/eqtl/scan_cis.hpp:15-66)
    def run_glm(self, scope, pthr):
        opt = self.opt
        works = []
        for gi, gene in enumerate(self.genes):
            loc = self.annot.get(gene) if opt.gff else None
            if scope == "cis" or scope == "trans":
                if loc is None:
                    continue
            elif opt.gff and loc is None and scope != "gw":
                continue
            works.append((gi, gene, loc))
        parallel_cis = scope == "cis" and opt.threads > 1 and bool(opt.gff)
        if parallel_cis:
            # the raw counts are checked before the sort (src/scan_cis.cpp:35-38)
            works = [w for w in works if R.looks_like_counts(self.Y[:, w[0]])]
            works.sort(key=lambda w: (w[2].chrom, w[2].tss))
        bim_chrom = [b[0] for b in self.bim]
        pairs, tops, summ = [], [], []
        pair_w, top_w = [], []  # position in `works` of each pair's / top's gene
        for wi, (gi, gene, loc) in enumerate(works):
            y = self.gene_y(gi)
            if not parallel_cis and not R.looks_like_counts(y):
                continue                                       # "skip non-count gene"
            ready = self.build_ready(y, need_k=False)
            if ready is None:
                continue
            keep, yk, Xk, _ = ready
            if scope == "cis":
                lo = max(loc.start - opt.window, 1)
                hi = loc.end + opt.window
                snps = [s_ for s_ in self.kept
                        if chrom_equal(bim_chrom[s_], loc.chrom) and lo <= self.bim[s_][3] <= hi]
            elif scope == "trans":
                snps = [s_ for s_ in self.kept if not self.in_cis(s_, loc)]
            else:
                snps = list(self.kept)
            s = Summary(gene)
            if loc is not None:
                s.chrom, s.tss = loc.chrom, loc.tss
            prep = R.prep_glm_nb(yk, Xk)
            acc = R.AcatAcc()
            best_p, best_row = 2.0, None
            cached = []
            if snps:
                G = self.dec.dosage[np.array(snps)][:, keep]
                af_sub, ok = R.subset_maf(G)
                st = R.test_glm_nb_many(prep, G)
                n = len(keep)
                for i, snp in enumerate(snps):
                    pv = st["p"][i]
                    if not ok[i] or not math.isfinite(pv):
                        continue
                    s.n_tested += 1
                    acc.add_many([pv])
                    acc.add_sensitivity([pv], [st["stat"][i]], None)
                    row = pair_row(gene, self.snp_meta(snp), _hit(st, i, af_sub[i]), n, loc, scope) + (
                        fmt(prep.phi), "1" if prep.converged else "0")
                    if pv <= pthr:
                        pairs.append(row)
                        pair_w.append(wi)
                        s.n_sig += 1
                    if pv < best_p:
                        best_p, best_row = pv, row
                    cached.append(G[i])
            s.acat = acc.p()
            s.acat_sens = acc.log10_sensitivity()
            if opt.perm > 0 and s.n_tested > 0:
                # parametric NB resampling of the null fit (include/eqtl/scan_cis.hpp:106-127)
                if (len(cached) - 1) * len(keep) > 25_000_000:
                    raise ValueError("cis perm: too many SNPs in cis window for gene " + gene)
                Ys = R.nb_resample(prep.mu, prep.phi, [R.perm_seed(opt.seed, b, gene) for b in range(opt.perm)])
                Gc = np.array(cached)
                T_perm, minps = [], []
                for b in range(opt.perm):
                    pv = R.test_glm_nb_many(R.prep_glm_nb(Ys[b], Xk), Gc)["p"]
                    pv = pv[np.isfinite(pv)]
                    minp = min(1.0, float(pv.min())) if pv.size else 1.0
                    T_perm.append(-math.log10(max(minp, 1e-300)))
                    minps.append(minp)
                s.p_emp = R.p_emp_count(-math.log10(max(best_p, 1e-300)), T_perm)
                if not opt.disable_beta_approx:
                    s.p_beta, s.s1, s.s2 = R.beta_approx_p(minps, best_p)
            if best_row is not None and best_p <= pthr and best_p <= 1.0:
                tops.append(best_row)
                top_w.append(wi)
            summ.append(s)
        if parallel_cis:
            pairs = per_thread_written(pairs, pair_w, opt.threads, len(works))
            tops = per_thread_written(tops, top_w, opt.threads, len(works))
        return pairs, tops, self.finish(summ)

    # -- permutations (include/eqtl/scan_cis.hpp:68-176, src/scan_perm.cpp:11-142) --
    def perm(self, model, s: Summary, gene, ready, cached, best_p, prep, lmm_basis=None):
        opt = self.opt
        keep, yk, Xk, _ = ready
        if model == "lm":
            base = prep.y_s
        else:
            Q, lam = lmm_basis
            Xb0 = prep.Xtil @ prep.chi0
            rt = prep.ytil - Xb0
            base = rt * np.sqrt(prep.dinv)
        Gc = np.array(cached)
        T_perm, minps = [], []
        for b in range(opt.perm):
            idx = R.shuffle_indices(len(base), R.perm_seed(opt.seed, b, gene))
            yb = base[np.array(idx)]
            if model == "lm":
                pb = R.prep_lm(yb, Xk)
                pv = R.test_lm_many(pb, Gc)["p"]
            else:
                r_perm = yb / np.sqrt(np.maximum(prep.dinv, 1e-12))
                yb = Q @ (Xb0 + r_perm)
                pb = R.prep_lmm(yb, Xk, Q, lam)
                pv = R.test_lmm_many(pb, Gc)["p"]
            pv = pv[np.isfinite(pv)]
            minp = min(1.0, float(pv.min())) if pv.size else 1.0
            T_perm.append(-math.log10(max(minp, 1e-300)))
            minps.append(minp)
        s.p_emp = R.p_emp_count(-math.log10(max(best_p, 1e-300)), T_perm)
        if not opt.disable_beta_approx:
            s.p_beta, s.s1, s.s2 = R.beta_approx_p(minps, best_p)
        self.last_perm_min_p = minps


def _p1(af):
    return {"beta": 0.0, "se": 0.0, "stat": 0.0, "p": 1.0, "r2": 0.0, "af": af}


def load_grm_sliced(prefix: str, samples: List[str]) -> np.ndarray:
    """load_grm_gcta + slice_grm, src/grm.cpp:10-45,80-108."""
    ids = []
    for ln in open(prefix + ".grm.id"):
        t = ln.split()
        if t:
            ids.append(t[1] if len(t) >= 2 else t[0])
    n = len(ids)
    buf = np.fromfile(prefix + ".grm.bin", dtype=np.float32, count=n * (n + 1) // 2).astype(np.float64)
    K = np.zeros((n, n))
    il = np.tril_indices(n)
    order = np.lexsort((il[1], il[0]))
    K[il[0][order], il[1][order]] = buf
    K = K + np.tril(K, -1).T
    pos = {s: i for i, s in enumerate(ids)}
    ix = np.array([pos[s] for s in samples])
    return K[np.ix_(ix, ix)]
