"""CPU restatement of the reference eqtl association-scan hot path (numpy).

TEST INFRASTRUCTURE ONLY. This module is the checker: tests/, the smoke
check and bench.py's CPU-baseline leg may call it; the product never does.
Every function cites the reference file:line it restates (paths relative to
the reference project root). Parity of this restatement is pinned against
outputs of the reference itself, built from its own sources by
oracle/Makefile (tests/golden/ holds those outputs and the script that
made them).

Arithmetic is FP64 like the reference. Sums run in numpy's order, so values
agree with the reference to ~1e-12 relative, not bit-for-bit; the integer
work (bed decode codes, missing counts, GRM N counts) is bit-exact.
"""
from __future__ import annotations

import math
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# PLINK .bed decode  (src/plink_bed.cpp:263-320, LUT :221-224)
# ---------------------------------------------------------------------------
_LUT = np.array([2, -1, 1, 0], dtype=np.int8)  # 00->2, 01->NA, 10->1, 11->0


def pass_maf(af, maf_min):
    """include/eqtl/util.hpp:61-64 (keep if maf_min <= af <= 1-maf_min)."""
    af = np.asarray(af, dtype=np.float64)
    if maf_min <= 0.0:
        return np.ones(af.shape, dtype=bool)
    return ~((af < maf_min) | (af > 1.0 - maf_min))


@dataclass
class Decoded:
    keep: np.ndarray       # bool [m]: SNP survives decode_row
    codes: np.ndarray      # int8 [m, n]: A1 count, -1 missing (all SNPs)
    dosage: np.ndarray     # float64 [m, n]: mean-imputed (all SNPs)
    n_miss: np.ndarray     # int32 [m]
    af: np.ndarray         # float64 [m]: mean(A1 count)/2 of non-missing


def decode_bed_rows(rows: np.ndarray, n_file: int, sample_col: Sequence[int], miss_hand: str,
                    max_miss: float, maf_min: float) -> Decoded:
    """PlinkBed::decode_row, src/plink_bed.cpp:263-320, vectorised over SNPs.

    rows: uint8 [m, ceil(n_file/4)] SNP-major bed bytes; sample_col maps the
    analysis order onto .fam columns (src/plink_bed.cpp:245-255)."""
    col = np.asarray(sample_col, dtype=np.int64)
    if np.any(col < 0) or np.any(col >= n_file):
        raise ValueError("sample_col out of range")
    byte = rows[:, col // 4]
    pair = (byte >> (2 * (col % 4)).astype(np.uint8)) & 3
    codes = _LUT[pair]
    miss = codes < 0
    n = col.size
    n_miss = miss.sum(1).astype(np.int32)
    n_ok = n - n_miss
    s = np.where(miss, 0, codes).sum(1).astype(np.float64)          # exact integer sum
    with np.errstate(divide="ignore", invalid="ignore"):
        mu = s / n_ok                                                # :299
        af = (s / n_ok) / 2.0                                        # :305
    keep = n_ok > 0                                                  # :292
    miss_frac = n_miss / float(n)
    keep &= ~(miss_frac > max_miss + 1e-15)                          # :295
    if miss_hand == "filter":
        keep &= n_miss == 0                                          # :297
    af = np.clip(np.nan_to_num(af, nan=0.0), 0.0, 1.0)               # :306-307
    keep &= ~((af < 1e-12) | (af > 1.0 - 1e-12))                     # :308
    keep &= pass_maf(af, maf_min)                                    # :309
    dosage = codes.astype(np.float64)
    if miss_hand == "impute":
        dosage = np.where(miss, mu[:, None], dosage)                 # :298-302
    else:
        dosage = np.where(miss, np.nan, dosage)
    return Decoded(keep, codes, dosage, n_miss, af)


# ---------------------------------------------------------------------------
# VCF GT records  (src/vcf_session.cpp:148-157 haploid contigs, :160-290
# parse_record, :294-305 for_each_snp with pass_maf)
# ---------------------------------------------------------------------------
def _vcf_haploid_chrom(chrom: str) -> bool:
    k = chrom
    if len(k) > 3 and k[:3].lower() == "chr":
        k = k[3:]
    return k in ("X", "x", "Y", "y", "M", "m", "MT", "mt", "Mt")


def read_vcf_gt(path: str):
    """Text VCF (plain or gzip): the biallelic records with a GT field as
    (chrom, pos, id, ref, alt, dosage[int8, -1 missing], haploid_call[bool]),
    plus the sample ids and the number of records that were not biallelic."""
    import gzip
    opener = gzip.open if open(path, "rb").read(2) == b"\x1f\x8b" else open
    samples, recs, n_multi = [], [], 0
    with opener(path, "rt") as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            if line.startswith("#CHROM"):
                samples = line.split("\t")[9:]
                continue
            if line.startswith("#"):
                continue
            fld = line.split("\t")
            alt = fld[4]
            if alt == "." or "," in alt:
                n_multi += 1
                continue
            keys = fld[8].split(":")
            if "GT" not in keys:
                continue
            gi = keys.index("GT")
            dos = np.empty(len(samples), np.int8)
            hap = np.zeros(len(samples), bool)
            for i, sf in enumerate(fld[9:9 + len(samples)]):
                sub = sf.split(":")
                gt = sub[gi] if gi < len(sub) else "."
                al = gt.replace("|", "/").split("/")[:2]
                if al[0] == "." or (len(al) > 1 and al[1] == "."):
                    dos[i] = -1
                    continue
                dos[i] = sum(int(a) for a in al)
                hap[i] = len(al) == 1
            recs.append((fld[0], int(fld[1]), "" if fld[2] == "." else fld[2], fld[3], alt, dos, hap))
    return samples, recs, n_multi


def _vcf_header_id(line: str):
    body = line[line.index("<") + 1:]
    if '"' in body:
        body = body[:body.index('"')]
    kv = dict(x.split("=", 1) for x in body.replace(">", ",").split(",") if "=" in x)
    return kv.get("ID"), kv.get("Type")


def _ds_value(text: str) -> float:
    """One FORMAT/DS value as htslib stores it (an FP32 number); '.', an
    unparseable or a non-finite value is missing (NaN)."""
    if text in ("", "."):
        return float("nan")
    try:
        v = float(np.float32(float(text.split(",")[0])))
    except ValueError:
        return float("nan")
    return v if np.isfinite(v) else float("nan")


def read_vcf_dosage(path: str):
    """Text VCF (plain or gzip) as parse_record reads it
    (src/vcf_session.cpp:66-68 DS detection, :193-258 DS / GT dosages):
    when the header defines an ID "DS", a record whose FORMAT has DS (declared
    Type=Float) takes each sample's DS value, other records their GT counts.
    Returns (samples, records, n_multi) with records (chrom, pos, id, ref, alt,
    dosage[float64, NaN missing], haploid_call[bool], used_ds)."""
    import gzip
    opener = gzip.open if open(path, "rb").read(2) == b"\x1f\x8b" else open
    samples, recs, n_multi = [], [], 0
    prefer_ds = ds_float = False
    with opener(path, "rt") as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            if line.startswith(("##INFO=<", "##FORMAT=<", "##FILTER=<")):
                hid, htype = _vcf_header_id(line)
                if hid == "DS":
                    prefer_ds = True
                    if line.startswith("##FORMAT=<"):
                        ds_float = htype == "Float"
                continue
            if line.startswith("#CHROM"):
                samples = line.split("\t")[9:]
                continue
            if line.startswith("#"):
                continue
            fld = line.split("\t")
            alt = fld[4]
            if alt == "." or "," in alt:
                n_multi += 1
                continue
            keys = fld[8].split(":")
            use_ds = prefer_ds and ds_float and "DS" in keys
            if not use_ds and "GT" not in keys:
                continue
            dos = np.full(len(samples), np.nan)
            hap = np.zeros(len(samples), bool)
            if use_ds:
                di = keys.index("DS")
                for i, sf in enumerate(fld[9:9 + len(samples)]):
                    sub = sf.split(":")
                    dos[i] = _ds_value(sub[di] if di < len(sub) else ".")
            else:
                gi = keys.index("GT")
                for i, sf in enumerate(fld[9:9 + len(samples)]):
                    sub = sf.split(":")
                    gt = sub[gi] if gi < len(sub) else "."
                    al = gt.replace("|", "/").split("/")[:2]
                    if al[0] in (".", "") or (len(al) > 1 and al[1] == "."):
                        continue
                    dos[i] = sum(int(a) for a in al)
                    hap[i] = len(al) == 1
            recs.append((fld[0], int(fld[1]), "" if fld[2] == "." else fld[2], fld[3], alt, dos, hap, use_ds))
    return samples, recs, n_multi


def decode_dosage_rows(ds: np.ndarray, sample_col: Sequence[int], miss_hand: str, max_miss: float,
                       maf_min: float) -> Decoded:
    """decode_bed_rows for FP32 dosage rows [m, n_file] (a value that is not
    finite is a missing call): the filters of src/plink_bed.cpp:292-309 with
    af = (sum / n_ok) / 2, the sums in FP64 in sample order, and mean
    imputation (src/vcf_session.cpp:270-279). `codes` holds -1 at missing
    calls and 0 elsewhere."""
    col = np.asarray(sample_col, dtype=np.int64)
    d = np.asarray(ds, dtype=np.float32)[:, col].astype(np.float64)
    miss = ~np.isfinite(d)
    n = col.size
    n_miss = miss.sum(1).astype(np.int32)
    n_ok = n - n_miss
    s = np.zeros(d.shape[0])
    dz = np.where(miss, 0.0, d)
    for i in range(n):                                               # sequential FP64 sums
        s += dz[:, i]
    with np.errstate(divide="ignore", invalid="ignore"):
        mu = s / n_ok
        af = (s / n_ok) / 2.0
    keep = n_ok > 0
    keep &= ~(n_miss / float(n) > max_miss + 1e-15)
    if miss_hand == "filter":
        keep &= n_miss == 0
    af = np.clip(np.nan_to_num(af, nan=0.0), 0.0, 1.0)
    keep &= ~((af < 1e-12) | (af > 1.0 - 1e-12))
    keep &= pass_maf(af, maf_min)
    dosage = np.where(miss, mu[:, None] if miss_hand == "impute" else np.nan, d)
    codes = np.where(miss, -1, 0).astype(np.int8)
    return Decoded(keep, codes, dosage, n_miss, af)


def vcf_keep(recs, sample_col: Sequence[int], max_miss: float, miss_filter: bool, maf_min: float) -> np.ndarray:
    """parse_record's filters over the analysis samples, then pass_maf on the
    ploidy-aware allele frequency (haploid contigs and haploid calls count one
    allele per call)."""
    col = np.asarray(sample_col, dtype=np.int64)
    keep = np.zeros(len(recs), bool)
    for r, rec in enumerate(recs):
        chrom, dos, hap = rec[0], rec[5], rec[6]
        d = dos[col]
        ok = d >= 0 if d.dtype.kind == "i" else np.isfinite(d)
        n_ok = int(ok.sum())
        n_miss = len(col) - n_ok
        if n_ok == 0:
            continue
        if n_miss / len(col) > max_miss + 1e-15:
            continue
        ploidy = np.where(_vcf_haploid_chrom(chrom) | hap[col], 1.0, 2.0)
        psum = float(ploidy[ok].sum())
        af = float(d[ok].sum()) / psum if psum > 0 else 0.0
        af = min(max(af, 0.0), 1.0)
        if af < 1e-12 or af > 1.0 - 1e-12:
            continue
        if miss_filter and n_miss > 0:
            continue
        if not pass_maf(af, maf_min):
            continue
        keep[r] = True
    return keep


def read_bed(prefix: str) -> Tuple[np.ndarray, int, list, list]:
    """Reads .fam/.bim/.bed like src/plink_bed.cpp:26-212 (no checks beyond the
    magic bytes). Returns (rows [m, nb], n_file, fam IIDs, bim records)."""
    fam = [ln.split()[1] for ln in open(prefix + ".fam") if ln.strip()]
    bim = []
    for ln in open(prefix + ".bim"):
        t = ln.split()
        if not t:
            continue
        bim.append((t[0], t[1], float(t[2]), int(t[3]), t[4], t[5]))
    raw = np.fromfile(prefix + ".bed", dtype=np.uint8)
    if raw[0] != 0x6C or raw[1] != 0x1B or raw[2] != 0x01:
        raise ValueError("bad bed magic")
    nb = (len(fam) + 3) // 4
    rows = raw[3:3 + nb * len(bim)].reshape(len(bim), nb)
    return rows, len(fam), fam, bim


# ---------------------------------------------------------------------------
# Student-t two-sided p  (src/util.cpp:209-264)
# ---------------------------------------------------------------------------
def _betacf(a, b, x):
    """Lentz continued fraction, src/util.cpp:209-241 (maxit 200, eps 3e-12)."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64); x = np.asarray(x, np.float64)
    fpmin = 1e-30
    qab = a + b; qap = a + 1.0; qam = a - 1.0
    c = np.ones_like(x)
    d = 1.0 - qab * x / qap
    d = np.where(np.abs(d) < fpmin, fpmin, d)
    d = 1.0 / d
    h = d.copy()
    done = np.zeros(x.shape, dtype=bool)
    for m in range(1, 201):
        m2 = 2 * m
        aa = m * (b - m) * x / ((qam + m2) * (a + m2))
        d_n = 1.0 + aa * d
        d_n = np.where(np.abs(d_n) < fpmin, fpmin, d_n)
        c_n = 1.0 + aa / c
        c_n = np.where(np.abs(c_n) < fpmin, fpmin, c_n)
        d_n = 1.0 / d_n
        h_n = h * d_n * c_n
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2))
        d_n2 = 1.0 + aa * d_n
        d_n2 = np.where(np.abs(d_n2) < fpmin, fpmin, d_n2)
        c_n2 = 1.0 + aa / c_n
        c_n2 = np.where(np.abs(c_n2) < fpmin, fpmin, c_n2)
        d_n2 = 1.0 / d_n2
        de = d_n2 * c_n2
        h_n = h_n * de
        upd = ~done
        d = np.where(upd, d_n2, d); c = np.where(upd, c_n2, c); h = np.where(upd, h_n, h)
        done |= upd & (np.abs(de - 1.0) < 3e-12)
        if done.all():
            break
    return h


def _lgamma(v):
    return np.vectorize(math.lgamma, otypes=[np.float64])(v)


def betai(a, b, x):
    """Regularised incomplete beta I_x(a,b), src/util.cpp:243-250."""
    a, b, x = np.broadcast_arrays(np.asarray(a, np.float64), np.asarray(b, np.float64),
                                  np.asarray(x, np.float64))
    out = np.full(x.shape, np.nan)
    edge = (x == 0) | (x == 1)
    out[edge] = x[edge]
    mid = (x > 0) & (x < 1)
    if mid.any():
        am, bm, xm = a[mid], b[mid], x[mid]
        lbeta = _lgamma(am) + _lgamma(bm) - _lgamma(am + bm)
        front = np.exp(np.log(xm) * am + np.log(1 - xm) * bm - lbeta) / am
        lo = xm < (am + 1) / (am + bm + 2)
        r = np.empty(xm.shape)
        if lo.any():
            r[lo] = front[lo] * _betacf(am[lo], bm[lo], xm[lo])
        hi = ~lo
        if hi.any():
            r[hi] = 1.0 - front[hi] * _betacf(bm[hi], am[hi], 1 - xm[hi]) * am[hi] / bm[hi]
        out[mid] = r
    return out


def p_from_t(t, df):
    """Two-sided Student-t p, src/util.cpp:259-264."""
    t = np.asarray(t, np.float64)
    df = np.broadcast_to(np.asarray(df, np.float64), t.shape)
    out = np.ones(t.shape)
    ok = np.isfinite(t) & (df > 0)
    if ok.any():
        x = df[ok] / (df[ok] + t[ok] * t[ok])
        out[ok] = np.clip(betai(0.5 * df[ok], 0.5, x), 0.0, 1.0)
    return out


def beta_cdf(x, a, b):
    """src/util.cpp:252-257."""
    if a <= 0 or b <= 0:
        return float("nan")
    if x <= 0:
        return 0.0
    if x >= 1:
        return 1.0
    return float(betai(a, b, x))


# ---------------------------------------------------------------------------
# Gene-level statistics (src/stats_extra.cpp:16-158, src/scan_common.cpp:201-217)
# ---------------------------------------------------------------------------
_PI_L = np.longdouble("3.14159265358979323846")


class AcatAcc:
    """AcatAcc::add/p, src/stats_extra.cpp:16-31 (long double tan sum)."""

    def __init__(self):
        self.tan_sum = np.longdouble(0)
        self.used = 0

    def add_many(self, p):
        p = np.asarray(p, np.float64)
        p = p[np.isfinite(p) & (p >= 0.0) & (p < 1.0 - 1e-12)]
        p = np.where(p <= 0.0, 1e-300, p)
        if p.size:
            self.tan_sum += np.sum(np.tan((np.longdouble(0.5) - p.astype(np.longdouble)) * _PI_L))
            self.used += int(p.size)

    def add_sensitivity(self, p, t, df):
        """Accumulates sum_j |d tan((0.5-p_j)pi) / d t_j| over the p's that
        enter the sum: the first-order amplification of an error in t into
        the ACAT statistic (pi (1+term^2) * 2 f_t(t; df))."""
        p = np.asarray(p, np.float64); t = np.asarray(t, np.float64)
        use = np.isfinite(p) & (p >= 0.0) & (p < 1.0 - 1e-12)
        if not use.any():
            return
        term = np.tan((0.5 - np.where(p[use] <= 0, 1e-300, p[use])) * np.pi)
        tt = t[use]
        if df is None:                                   # normal statistic (GLM score test)
            logf = -0.5 * math.log(2 * math.pi) - 0.5 * tt * tt
        else:
            logf = (math.lgamma((df + 1) / 2) - math.lgamma(df / 2) - 0.5 * math.log(df * math.pi)
                    - (df + 1) / 2 * np.log1p(tt * tt / df))
        self.sens = getattr(self, "sens", 0.0) + float(np.sum(np.pi * (1 + term * term) * 2 * np.exp(logf)))

    def log10_sensitivity(self) -> float:
        """|d log10(acat_p) / d t| bound per unit error in every t."""
        if self.used == 0 or not getattr(self, "sens", 0.0):
            return 0.0
        T = float(self.tan_sum / np.longdouble(self.used))
        ac = max(self.p(), 1e-300)
        return self.sens / self.used / (np.pi * (1 + T * T)) / (ac * math.log(10))

    def p(self) -> float:
        if self.used == 0:
            return 1.0
        T = self.tan_sum / np.longdouble(self.used)
        ac = 0.5 - float(np.arctan(T) / _PI_L)
        return min(max(ac, 0.0), 1.0)


def p_emp_count(T_obs: float, T_perm: Sequence[float]) -> float:
    """src/stats_extra.cpp:39-46."""
    ge = sum(1 for t in T_perm if t >= T_obs)
    return (1.0 + ge) / (1.0 + len(T_perm))


def beta_fit_mm(x: np.ndarray):
    """src/stats_extra.cpp:79-91."""
    if x.size < 2:
        return None
    mean = float(np.sum(x)) / x.size
    var = float(np.sum((x - mean) ** 2)) / (x.size - 1)
    if var <= 0 or mean <= 0 or mean >= 1:
        return None
    t = mean * (1.0 - mean) / var - 1.0
    if t <= 0:
        return None
    return mean * t, (1.0 - mean) * t


def _nm_minimise(f, x0, step, tol=0.01, maxit=1000):
    """Nelder-Mead in the `nmsimplex2` form (reflect -1, expand -2, contract
    0.5, shrink to best; size = RMS vertex distance from the centroid) used by
    src/stats_extra.cpp:95-126 through GSL."""
    n = len(x0)
    xs = [np.array(x0, float)] + [np.array(x0, float) + step[i] * np.eye(n)[i] for i in range(n)]
    ys = [f(v) for v in xs]
    P = n + 1

    def center_size():
        c = sum(xs) / P
        return c, math.sqrt(sum(float(np.sum((v - c) ** 2)) for v in xs) / P)

    c, size = center_size()
    it = 0
    status_ok = False
    while True:
        it += 1
        hi = lo = 0; s_hi = 1
        dhi = dlo = ys[0]; ds_hi = ys[1]
        for i in range(1, P):
            v = ys[i]
            if v < dlo:
                dlo = v; lo = i
            elif v > dhi:
                ds_hi = dhi; s_hi = hi; dhi = v; hi = i
            elif v > ds_hi:
                ds_hi = v; s_hi = i

        def move(coeff, corner):
            alpha = (1 - coeff) * P / (P - 1.0)
            beta = (P * coeff - 1.0) / (P - 1.0)
            return alpha * c + beta * xs[corner]

        xr = move(-1.0, hi); vr = f(xr)
        if math.isfinite(vr) and vr < ys[lo]:
            xe = move(-2.0, hi); ve = f(xe)
            if math.isfinite(ve) and ve < ys[lo]:
                xs[hi], ys[hi] = xe, ve
            else:
                xs[hi], ys[hi] = xr, vr
            c, size = center_size()
        elif (not math.isfinite(vr)) or vr > ys[s_hi]:
            if math.isfinite(vr) and vr <= ys[hi]:
                xs[hi], ys[hi] = xr, vr
                c, size = center_size()
            xk = move(0.5, hi); vk = f(xk)
            if math.isfinite(vk) and vk <= ys[hi]:
                xs[hi], ys[hi] = xk, vk
            else:
                for i in range(P):
                    if i != lo:
                        xs[i] = 0.5 * (xs[i] + xs[lo])
                        ys[i] = f(xs[i])
            c, size = center_size()
        else:
            xs[hi], ys[hi] = xr, vr
            c, size = center_size()
        best = int(np.argmin(ys))
        if size < tol:
            status_ok = True
            break
        if it >= maxit:
            break
    return xs[best], status_ok


def beta_approx_p(perm_min_p: Sequence[float], obs_min_p: float):
    """src/stats_extra.cpp:131-158. Returns (p_beta, shape1, shape2)."""
    x = np.array([v for v in perm_min_p if math.isfinite(v) and 0.0 < v < 1.0])
    nan = float("nan")
    if x.size < 10:
        return nan, nan, nan
    mm = beta_fit_mm(x)
    if mm is None:
        return nan, nan, nan
    s1, s2 = mm
    xv = np.where(x >= 1.0, 0.99999999, x)
    S1 = float(np.sum(np.log(xv))); S2 = float(np.sum(np.log(1.0 - xv))); N = float(xv.size)

    def nll(v):
        a, b = float(v[0]), float(v[1])
        if not (0.1 <= a <= 10.0 and 5.0 <= b <= 1e6):
            return 1e300
        lnb = math.lgamma(a) + math.lgamma(b) - math.lgamma(a + b)
        return -((a - 1.0) * S1 + (b - 1.0) * S2 - N * lnb)

    ok = s1 > 0 and s2 > 0
    if ok:
        xb, conv = _nm_minimise(nll, [s1, s2], [s1 / 10.0, s2 / 10.0])
        a, b = float(xb[0]), float(xb[1])
        if conv and math.isfinite(a) and math.isfinite(b) and 0.1 <= a <= 10.0 and 5.0 <= b <= 1e6:
            s1, s2 = a, b
    o = min(max(obs_min_p, 1e-300), 1.0 - 1e-16)
    pb = beta_cdf(o, s1, s2)
    return (pb if math.isfinite(pb) else nan), s1, s2


def bh_adjust(acat: Sequence[float]) -> np.ndarray:
    """src/scan_common.cpp:201-217."""
    a = np.asarray(acat, np.float64)
    m = a.size
    q = np.empty(m)
    idx = np.argsort(a, kind="stable")
    prev = 1.0
    for rank in range(m, 0, -1):
        j = idx[rank - 1]
        v = a[j] * m / rank
        v = min(v, prev, 1.0)
        q[j] = v
        prev = v
    return q


# ---------------------------------------------------------------------------
# Per-SNP gate on the analysis subset  (src/scan_common.cpp:133-151)
# ---------------------------------------------------------------------------
def subset_maf(G: np.ndarray):
    """Returns (af_sub [m], ok [m]) for dosage rows G [m, n]."""
    n = G.shape[1]
    s = G.sum(1); s2 = (G * G).sum(1)
    af = np.clip((s / n) / 2.0, 0.0, 1.0)
    maf = np.where(af > 0.5, 1.0 - af, af)
    var = s2 / n - (s / n) ** 2
    ok = np.isfinite(s) & ~(maf < 1e-12) & ~(var < 1e-12)
    return af, ok


# ---------------------------------------------------------------------------
# LM  (src/model_lm.cpp:19-57, src/scan_trans_lm.cpp:11-36)
# ---------------------------------------------------------------------------
@dataclass
class PrepLm:
    y_s: np.ndarray
    X: np.ndarray
    XtX_inv: np.ndarray
    yty: float
    n: int
    p: int


def prep_lm(y, X) -> PrepLm:
    XtX = X.T @ X
    XtX_inv = np.linalg.solve(XtX, np.eye(X.shape[1]))
    beta = XtX_inv @ (X.T @ y)
    y_s = y - X @ beta
    return PrepLm(y_s, X, XtX_inv, float(y_s @ y_s), len(y), X.shape[1])


def lm_stats(gtg, gty, yty, n, p):
    """hit_from_gty / test_lm arithmetic, vectorised. Returns dict of arrays."""
    gtg = np.asarray(gtg, float); gty = np.asarray(gty, float)
    shape = np.broadcast(gtg, gty, yty).shape
    gtg = np.broadcast_to(gtg, shape); gty = np.broadcast_to(gty, shape)
    yty = np.broadcast_to(np.asarray(yty, float), shape)
    out = {k: np.zeros(shape) for k in ("beta", "se", "stat", "r2")}
    out["p"] = np.ones(shape)
    df = n - p - 1
    ok = ~(gtg < 1e-12)
    if df <= 0:
        return out
    with np.errstate(divide="ignore", invalid="ignore"):
        beta = np.where(ok, gty / gtg, 0.0)
        rss = yty - beta * gty
        s2 = np.maximum(rss / df, 0.0)
        se = np.where(ok, np.sqrt(s2 / gtg), 0.0)
        stat = np.where(se > 0, beta / se, 0.0)
        r2 = np.where(yty > 0, 1.0 - rss / yty, 0.0)
    out["beta"] = np.where(ok, beta, 0.0); out["se"] = se; out["stat"] = np.where(ok, stat, 0.0)
    out["r2"] = np.where(ok, r2, 0.0)
    out["p"] = np.where(ok, p_from_t(out["stat"], df), 1.0)
    return out


def test_lm_many(prep: PrepLm, G: np.ndarray):
    """test_lm over dosage rows G [m, n] (src/model_lm.cpp:32-57)."""
    Xt_g = G @ prep.X
    g_s = G - (Xt_g @ prep.XtX_inv.T) @ prep.X.T
    gtg = np.einsum("ij,ij->i", g_s, g_s)
    gty = g_s @ prep.y_s
    return lm_stats(gtg, gty, prep.yty, prep.n, prep.p)


# ---------------------------------------------------------------------------
# NB GLM  (src/model_glm.cpp:13-132; looks_like_counts src/model_lm.cpp:8-17;
# pnorm_two_sided src/util.cpp:116-123)
# ---------------------------------------------------------------------------
def looks_like_counts(y) -> bool:
    y = np.asarray(y, np.float64)
    f = y[np.isfinite(y)]
    if f.size == 0:
        return False
    return bool(np.all(f >= 0) and np.all(np.abs(f - np.floor(f)) <= 1e-8))


def pnorm_two_sided(z):
    """erfc(|z| / sqrt(2)) clipped to [0, 1]; 1 for a non-finite z."""
    z = np.asarray(z, np.float64)
    from scipy.special import erfc
    p = np.where(np.isfinite(z), erfc(np.abs(z) / math.sqrt(2.0)), 1.0)
    return np.clip(p, 0.0, 1.0)


@dataclass
class PrepGlm:
    y: np.ndarray
    X: np.ndarray
    mu: np.ndarray
    w: np.ndarray          # null working weights mu / (1 + phi mu)
    r: np.ndarray          # (y - mu) / (1 + phi mu)
    XtWX_inv: np.ndarray
    phi: float
    converged: bool
    n: int


def _nb_mom_phi(y, mu, df):
    m = np.maximum(mu, 1e-8)
    num = float(np.sum(((y - m) * (y - m) - m) / (m * m)))
    return max(1e-8, num / max(1, df))


def nb_irls(y, X, phi):
    """nb_irls (src/model_glm.cpp:28-72) with estimate_phi: IRLS at fixed phi
    (up to 50 rounds, until max |beta change| < 1e-6), then phi by moments,
    until phi moves less than 1e-6 max(1, phi) (up to 10 rounds). Returns
    (phi, beta, mu, converged); converged is False only when X'WX cannot be
    factorised."""
    n, p = X.shape
    df = max(1, n - p)
    beta = np.zeros(p)
    mu = np.maximum(y, 0.1)
    for _ in range(10):
        for _ in range(50):
            m = np.maximum(mu, 1e-8)
            var = m + phi * m * m
            w = (m * m) / np.maximum(var, 1e-12)
            z = np.log(m) + (y - m) / m
            XtWX = X.T @ (w[:, None] * X)
            try:
                np.linalg.cholesky(XtWX)
            except np.linalg.LinAlgError:
                return phi, beta, mu, False
            beta_new = np.linalg.solve(XtWX, X.T @ (w * z))
            mu_new = np.exp(X @ beta_new)
            diff = float(np.max(np.abs(beta_new - beta)))
            beta, mu = beta_new, mu_new
            if diff < 1e-6:
                break
        phi_new = _nb_mom_phi(y, mu, df)
        if abs(phi_new - phi) < 1e-6 * max(1.0, phi):
            return phi_new, beta, mu, True
        phi = phi_new
    return phi, beta, mu, True


def prep_glm_nb(y, X) -> PrepGlm:
    """prep_glm_nb (src/model_glm.cpp:74-96): the null NB fit from phi = 1."""
    y = np.asarray(y, np.float64)
    if not looks_like_counts(y):
        raise ValueError("glm (NB) requires non-negative integer counts")
    phi, _, mu, conv = nb_irls(y, X, 1.0)
    m = np.maximum(mu, 1e-8)
    w = m / (1.0 + phi * m)
    XtWX_inv = np.linalg.solve(X.T @ (w[:, None] * X), np.eye(X.shape[1]))
    r = (y - mu) / (1.0 + phi * mu)
    return PrepGlm(y, X, mu, w, r, XtWX_inv, phi, conv, y.size)


def test_glm_nb_many(prep: PrepGlm, G: np.ndarray):
    """test_glm_nb (src/model_glm.cpp:98-132) for dosage rows G [m, n]: the
    score test at beta_g = 0 with phi fixed, U = g'r, info = g'Wg -
    (X'Wg)' (X'WX)^-1 (X'Wg); beta = U / info, se = 1 / sqrt(info), stat =
    U / sqrt(info), p two-sided normal. p is NaN for a null fit that did not
    converge and 1 (the rest 0) for gvar or info below 1e-12."""
    G = np.atleast_2d(np.asarray(G, np.float64))
    m = G.shape[0]
    out = {k: np.zeros(m) for k in ("beta", "se", "stat", "p", "r2")}
    if not prep.converged:
        out["p"][:] = np.nan
        return out
    out["p"][:] = 1.0
    gvar = (G * G).mean(1) - G.mean(1) ** 2
    U = G @ prep.r
    XtWg = (G * prep.w[None, :]) @ prep.X
    info = np.einsum("ij,ij->i", G * prep.w[None, :], G) - np.einsum("ij,jk,ik->i", XtWg, prep.XtWX_inv, XtWg)
    ok = ~(gvar < 1e-12) & ~(info < 1e-12)
    si = np.sqrt(np.where(ok, info, 1.0))
    out["beta"] = np.where(ok, U / np.where(ok, info, 1.0), 0.0)
    out["se"] = np.where(ok, 1.0 / si, 0.0)
    out["stat"] = np.where(ok, U / si, 0.0)
    out["p"] = np.where(ok, pnorm_two_sided(out["stat"]), 1.0)
    return out


# ---------------------------------------------------------------------------
# LMM  (src/model_lmm.cpp:10-223, src/scan_trans_lmm.cpp:11-70)
# ---------------------------------------------------------------------------
_EIGSOLVE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "eigsolve")


def sparsify_grm(K, thr):
    """sparsify_grm (src/model_lmm.cpp:88-104): off-diagonal entries below
    thr in magnitude set to 0 (the --fast approximation)."""
    K = np.array(K, dtype=np.float64, copy=True)
    small = np.abs(K) < thr
    np.fill_diagonal(small, False)
    K[small] = 0.0
    return K


def make_lmm_basis(K):
    """src/model_lmm.cpp:106-113. Uses the reference's own eigensolver (Eigen,
    via oracle/_ref/eigsolve) when it has been built, so eigenvector signs
    match the reference binary; numpy's eigh otherwise (signs may differ,
    which only matters for LMM permutations)."""
    if os.path.exists(_EIGSOLVE):
        return eigen_basis_ref(K)
    lam, Q = np.linalg.eigh(K)
    return Q, np.maximum(lam, 0.0)


def eigen_basis_ref(K):
    n = K.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fi, fo = os.path.join(td, "k.bin"), os.path.join(td, "q.bin")
        with open(fi, "wb") as f:
            f.write(np.int64(n).tobytes())
            f.write(np.ascontiguousarray(K, dtype=np.float64).tobytes())
        subprocess.run([_EIGSOLVE, fi, fo], check=True)
        buf = np.fromfile(fo, dtype=np.float64)
    lam = buf[:n]
    Q = buf[n:].reshape(n, n).T  # column-major -> [row, col]
    return np.ascontiguousarray(Q), lam


def reml_negll(delta, ytil, Xtil, lam, df):
    """src/model_lmm.cpp:10-37."""
    v = np.maximum(delta * lam + 1.0, 1e-12)
    dinv = 1.0 / v
    logdet_d = float(np.sum(np.log(v)))
    XtDX = (Xtil * dinv[:, None]).T @ Xtil
    XtDy = Xtil.T @ (dinv * ytil)
    try:
        L = np.linalg.cholesky(XtDX)
    except np.linalg.LinAlgError:
        return 1e300
    beta = np.linalg.solve(XtDX, XtDy)
    q = float(ytil @ (dinv * ytil) - XtDy @ beta)
    if q <= 0:
        q = 1e-12
    sigma2 = q / df
    logdet_x = 2.0 * float(np.sum(np.log(np.diag(L))))
    return 0.5 * (df * math.log(sigma2) + logdet_d + logdet_x)


def optimize_delta(ytil, Xtil, lam):
    """Grid 1e-5..1e5 x2, 40 golden-section steps, <=8 Newton steps
    (src/model_lmm.cpp:39-86)."""
    n, p = Xtil.shape
    df = n - p
    if df <= 0:
        return 1.0
    f = lambda d: reml_negll(d, ytil, Xtil, lam, df)
    best_d = 1.0
    best_ll = f(1.0)
    d = 1e-5
    while d <= 1e5:
        v = f(d)
        if v < best_ll:
            best_ll = v; best_d = d
        d *= 2.0
    lo, hi = best_d / 4.0, best_d * 4.0
    lo = max(lo, 1e-8); hi = min(hi, 1e6)
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    for _ in range(40):
        m1 = hi - (hi - lo) / phi
        m2 = lo + (hi - lo) / phi
        if f(m1) < f(m2):
            hi = m2
        else:
            lo = m1
    d = 0.5 * (lo + hi)
    cur = f(d)
    for _ in range(8):
        h = max(d * 1e-4, 1e-9)
        fm = f(d - h); fp = f(d + h)
        g1 = (fp - fm) / (2.0 * h)
        g2 = (fp - 2.0 * cur + fm) / (h * h)
        if not (g2 > 1e-12):
            break
        step = g1 / g2
        dn = d - step
        if not (1e-8 < dn < 1e6):
            break
        vn = f(dn)
        if not (vn < cur):
            break
        d = dn; cur = vn
        if abs(step) < d * 1e-8:
            break
    return d


@dataclass
class PrepLmm:
    ytil: np.ndarray
    Xtil: np.ndarray
    lam: np.ndarray
    Q: np.ndarray
    dinv: np.ndarray
    delta: float
    rss_null: float
    chi0: np.ndarray
    A00: np.ndarray
    n: int
    p: int


def prep_lmm(y, X, Q, lam, delta=None) -> PrepLmm:
    """src/model_lmm.cpp:124-153. `delta` given: the null fit at that delta
    instead of the REML optimum (for checks at another optimiser's delta)."""
    ytil = Q.T @ y
    Xtil = Q.T @ X
    if delta is None:
        delta = optimize_delta(ytil, Xtil, lam)
    dinv = 1.0 / np.maximum(delta * lam + 1.0, 1e-12)
    A00 = (Xtil * dinv[:, None]).T @ Xtil
    Dy = dinv * ytil
    XtDy0 = Xtil.T @ Dy
    y_dy = float(ytil @ Dy)
    chi0 = np.linalg.solve(A00, XtDy0)
    rss_null = max(y_dy - float(XtDy0 @ chi0), 0.0)
    return PrepLmm(ytil, Xtil, lam, Q, dinv, delta, rss_null, chi0, A00, len(y), X.shape[1])


def lmm_stats_gtil(prep: PrepLmm, Gtil: np.ndarray):
    """Bordered-Schur fixed-delta Wald test on rotated dosages Gtil [m, n]
    (src/scan_trans_lmm.cpp:11-40 == src/model_lmm.cpp:160-201)."""
    Dg = Gtil * prep.dinv[None, :]
    gg = np.einsum("ij,ij->i", Dg, Gtil)
    a = Dg @ prep.Xtil                       # [m, p]
    yg = Dg @ prep.ytil
    u = np.linalg.solve(prep.A00, a.T).T
    S = gg - np.einsum("ij,ij->i", a, u)
    df = prep.n - prep.p - 1
    m = Gtil.shape[0]
    out = {k: np.zeros(m) for k in ("beta", "se", "stat", "r2")}
    out["p"] = np.ones(m)
    ok = ~(gg < 1e-12) & ~(S <= 1e-15)
    with np.errstate(divide="ignore", invalid="ignore"):
        bg = (yg - a @ prep.chi0) / S
        q = np.maximum(prep.rss_null - S * bg * bg, 0.0)
        sigma2 = q / df if df > 0 else np.ones(m)
        se = np.sqrt(np.maximum(sigma2 / S, 0.0))
        stat = np.where(se > 0, bg / se, 0.0)
        r2 = np.maximum(0.0, 1.0 - q / prep.rss_null) if prep.rss_null > 1e-15 else np.zeros(m)
    out["beta"] = np.where(ok, bg, 0.0)
    out["se"] = np.where(ok, se, 0.0)
    out["stat"] = np.where(ok, stat, 0.0)
    out["r2"] = np.where(ok, r2, 0.0)
    out["p"] = np.where(ok, p_from_t(out["stat"], df), 1.0)
    return out


def lmm_stats_gtil_genes(preps, Gtil: np.ndarray):
    """lmm_stats_gtil for several genes that share the eigenbasis, on the
    same rotated dosages Gtil [m, n]: the same arithmetic
    (src/scan_trans_lmm.cpp:11-40), with gg, a and yg of all genes formed as
    matrix products. Returns dict of [m, len(preps)] arrays."""
    W = np.column_stack([pr.dinv for pr in preps])             # [n, G]
    gg = (Gtil * Gtil) @ W                                      # [m, G]
    yg = Gtil @ (W * np.column_stack([pr.ytil for pr in preps]))
    m, G = Gtil.shape[0], len(preps)
    out = {k: np.zeros((m, G)) for k in ("beta", "se", "stat", "r2")}
    out["p"] = np.ones((m, G))
    for j, pr in enumerate(preps):
        a = Gtil @ (pr.Xtil * pr.dinv[:, None])                 # [m, p]
        u = np.linalg.solve(pr.A00, a.T).T
        S = gg[:, j] - np.einsum("ij,ij->i", a, u)
        df = pr.n - pr.p - 1
        ok = ~(gg[:, j] < 1e-12) & ~(S <= 1e-15)
        with np.errstate(divide="ignore", invalid="ignore"):
            bg = (yg[:, j] - a @ pr.chi0) / S
            q = np.maximum(pr.rss_null - S * bg * bg, 0.0)
            sigma2 = q / df if df > 0 else np.ones(m)
            se = np.sqrt(np.maximum(sigma2 / S, 0.0))
            stat = np.where(se > 0, bg / se, 0.0)
            r2 = np.maximum(0.0, 1.0 - q / pr.rss_null) if pr.rss_null > 1e-15 else np.zeros(m)
        out["beta"][:, j] = np.where(ok, bg, 0.0)
        out["se"][:, j] = np.where(ok, se, 0.0)
        out["stat"][:, j] = np.where(ok, stat, 0.0)
        out["r2"][:, j] = np.where(ok, r2, 0.0)
        out["p"][:, j] = np.where(ok, p_from_t(out["stat"][:, j], df), 1.0)
    return out


def test_lmm_many(prep: PrepLmm, G: np.ndarray):
    """test_lmm over raw dosage rows G [m, n] (rotates each row, :173)."""
    return lmm_stats_gtil(prep, G @ prep.Q)


# ---------------------------------------------------------------------------
# GRM  (src/grm.cpp:113-224, write :47-78)
# ---------------------------------------------------------------------------
def compute_grm(dosage: np.ndarray, miss: np.ndarray):
    """dosage [m, n] mean-imputed rows of the SNPs decode kept; miss [m, n]
    bool missing mask. Returns (K [n, n], N_packed int32 [n(n+1)/2], m_used)."""
    mu = dosage.mean(1)
    p = mu / 2.0
    use = ~((p < 1e-8) | (p > 1.0 - 1e-8))
    sd = np.sqrt(2.0 * p * (1.0 - p))
    use &= ~(sd < 1e-12)
    m = int(use.sum())
    if m == 0:
        raise ValueError("no SNPs for GRM")
    n = dosage.shape[1]
    A = np.zeros((n, n))
    joint = np.zeros((n, n))  # integer counts, exact in FP64
    ui = np.nonzero(use)[0]
    for c0 in range(0, ui.size, 16384):  # in SNP blocks, to bound the memory
        u = ui[c0:c0 + 16384]
        Z = (dosage[u] - mu[u, None]) / sd[u, None]
        A += Z.T @ Z
        M = miss[u].astype(np.float64)
        joint += M.T @ M
    sub_miss = miss[use].sum(0).astype(np.int64)
    joint = np.rint(joint).astype(np.int64)
    subN = m - sub_miss[:, None] - sub_miss[None, :] + joint
    np.fill_diagonal(subN, m - sub_miss)
    with np.errstate(divide="ignore", invalid="ignore"):
        K = np.where(subN > 0, A / subN, 0.0)
    il = np.tril_indices(n)
    # row-major lower triangle incl. diagonal: (i, j<=i)
    order = np.lexsort((il[1], il[0]))
    N_packed = subN[il[0][order], il[1][order]].astype(np.int32)
    return K, N_packed, m


def grm_lower_f32(K: np.ndarray) -> np.ndarray:
    n = K.shape[0]
    il = np.tril_indices(n)
    order = np.lexsort((il[1], il[0]))
    return K[il[0][order], il[1][order]].astype(np.float32)


# ---------------------------------------------------------------------------
# Permutation indices: std::mt19937 + libstdc++ std::shuffle
# (include/eqtl/scan_cis.hpp:106-111, src/scan_perm.cpp:84-88)
# ---------------------------------------------------------------------------
def fnv1a(s: str) -> int:
    """include/eqtl/util.hpp:51-58."""
    h = 14695981039346656037
    for c in s.encode():
        h ^= c
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h & 0xFFFFFFFF


class _MT19937:
    """Standard 32-bit Mersenne Twister with init_genrand seeding (the
    std::mt19937(value) constructor)."""

    def __init__(self, seed: int):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            self.mt[i] = (1812433253 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.idx = 624

    def __call__(self) -> int:
        if self.idx >= 624:
            mt = self.mt
            for i in range(624):
                y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
                mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
            self.idx = 0
        y = self.mt[self.idx]
        self.idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def _uniform_int(g: _MT19937, lo: int, hi: int) -> int:
    """libstdc++ uniform_int_distribution for a 32-bit engine: Lemire's
    nearly-divisionless downscale (multiply by range, reject low words below
    -range % range)."""
    rng = hi - lo + 1
    if rng == 1 << 32:
        return lo + g()
    prod = g() * rng
    low = prod & 0xFFFFFFFF
    if low < rng:
        thr = ((1 << 32) - rng) % rng
        while low < thr:
            prod = g() * rng
            low = prod & 0xFFFFFFFF
    return lo + (prod >> 32)


def shuffle_indices(n: int, seed: int) -> List[int]:
    """iota(n) shuffled by std::shuffle(first, last, std::mt19937(seed)) as
    libstdc++ implements it: when (2^32-1)/n >= n, swap positions are drawn
    two at a time from one uniform draw over [0, b*(b+1))."""
    idx = list(range(n))
    if n <= 1:
        return idx
    g = _MT19937(seed)
    urng_range = 0xFFFFFFFF
    if urng_range // n >= n:
        i = 1
        if n % 2 == 0:
            j = _uniform_int(g, 0, 1)
            idx[i], idx[j] = idx[j], idx[i]
            i += 1
        while i != n:
            b0 = i + 1
            x = _uniform_int(g, 0, b0 * (b0 + 1) - 1)
            p1, p2 = x // (b0 + 1), x % (b0 + 1)
            idx[i], idx[p1] = idx[p1], idx[i]
            i += 1
            idx[i], idx[p2] = idx[p2], idx[i]
            i += 1
        return idx
    for i in range(1, n):
        j = _uniform_int(g, 0, i)
        idx[i], idx[j] = idx[j], idx[i]
    return idx


def perm_seed(seed_opt: int, b: int, gene: str) -> int:
    base = seed_opt if seed_opt >= 0 else 1
    return (base + b * 9973 + fnv1a(gene)) & 0xFFFFFFFF


def nb_resample(mu: np.ndarray, phi: float, seeds: Sequence[int]) -> np.ndarray:
    """The reference's GLM permutation phenotypes (include/eqtl/scan_cis.hpp:
    106-127) drawn by the standard library itself (oracle/_ref/nbresample):
    one row of counts per seed."""
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "nbresample")
    inp = f"{len(mu)} {phi!r}\n" + " ".join(repr(float(m)) for m in mu) + f"\n{len(seeds)}\n" + \
        " ".join(str(int(s)) for s in seeds) + "\n"
    out = subprocess.run([exe], input=inp, check=True, capture_output=True, text=True).stdout
    return np.array([[float(v) for v in ln.split()] for ln in out.strip().split("\n")])


# ---------------------------------------------------------------------------
# PEER VB factor analysis of the fission subcommand (src/fission.cpp:104-275)
# ---------------------------------------------------------------------------
def std_normal_draws(seed: int, count: int) -> np.ndarray:
    """The standard library's std::normal_distribution sequence from
    std::mt19937(seed), read from oracle/_ref/stdnormal (built by
    oracle/Makefile from oracle/shim/stdnormal.cpp)."""
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "stdnormal")
    out = subprocess.run([exe, str(seed), str(count)], check=True, capture_output=True, text=True).stdout
    return np.array([float(v) for v in out.split()], dtype=np.float64)


def peer_start(seed: int, n: int, G: int, k: int):
    """peer_factors' starting values (src/fission.cpp:226-236): X [n, k] then
    W [G, k], both filled column by column from one normal sequence."""
    z = std_normal_draws(seed, n * k + G * k)
    X0 = z[: n * k].reshape(k, n).T.copy()
    W0 = z[n * k:].reshape(k, G).T.copy()
    return X0, W0


def peer_factors(Y_raw: np.ndarray, k: int, max_iter: int, tol: float, X0: np.ndarray, W0: np.ndarray):
    """peer_factors (src/fission.cpp:203-275) from given starting values:
    genes centred (NaN -> 0), ARD/noise priors (0.001, 0.1) / (0.1, 10),
    W, Alpha, X, Eps updates in that order, stop when the mean squared
    residual moves by less than 1e-8 or `tol`. Returns (X [n, k], iterations)."""
    Y = np.array(Y_raw, dtype=np.float64, copy=True)
    n, G = Y.shape
    for j in range(G):
        fin = ~np.isnan(Y[:, j])
        mean = Y[fin, j].mean() if fin.any() else 0.0
        Y[:, j] = np.where(fin, Y[:, j] - mean, 0.0)
    pa_A, pb_A, pa_E, pb_E = 0.001, 0.1, 0.1, 10.0
    X = X0.copy()
    W = W0.copy()
    Eps = np.full(G, pa_E / pb_E)
    XE2S = n * np.eye(k) + X.T @ X
    Alpha = (pa_A + 0.5 * G) / (pb_A + 0.5 * np.zeros(k))
    b1 = (Y * Y + 0.01).sum(0)
    last = np.finfo(np.float64).max
    it = 0
    for it in range(1, max_iter + 1):
        XtY = X.T @ Y
        covs = np.empty((G, k, k))
        for d in range(G):
            M = np.diag(Alpha) + Eps[d] * XE2S
            covs[d] = np.linalg.solve(M, np.eye(k))
            W[d] = np.linalg.solve(M, XtY[:, d]) * Eps[d]
        E2 = covs + W[:, :, None] * W[:, None, :]
        W_E2S = E2.sum(0)
        W_Xprec = (Eps[:, None, None] * E2).sum(0)
        Alpha = (pa_A + 0.5 * G) / (pb_A + 0.5 * np.diag(W_E2S))
        Xcov = np.linalg.solve(W_Xprec + np.eye(k), np.eye(k))
        X = Y @ (W * Eps[:, None]) @ Xcov
        XE2S = n * Xcov + X.T @ X
        b2 = (XtY.T * W).sum(1)
        b3 = np.einsum("kl,dkl->d", XE2S, E2)
        Eps = (pa_E + 0.5 * n) / np.maximum(pb_E + 0.5 * (b1 - 2.0 * b2 + b3), 1e-10)
        res = float(np.mean((Y - X @ W.T) ** 2))
        if abs(last - res) < 1e-8 or abs(last - res) < tol:
            break
        last = res
    return X, it


def fission_residualize(Y1: np.ndarray, X: np.ndarray) -> np.ndarray:
    """src/fission.cpp:331-344: per gene, values that are not finite take
    the gene's mean, then the least-squares fit on the covariates X (with
    intercept) is removed."""
    out = np.empty_like(Y1)
    for j in range(Y1.shape[1]):
        y = Y1[:, j].copy()
        fin = np.isfinite(y)
        y[~fin] = y[fin].mean() if fin.any() else 0.0
        b = np.linalg.solve(X.T @ X, X.T @ y)
        out[:, j] = y - X @ b
    return out
