"""ctypes binding of libeqtl_cuda (include/eqtl_b200.h).

This is the Python view of the C ABI used by the tests and the benchmark.
It loads the in-tree eqtl_b200/lib/libeqtl_cuda.so and raises if it is
missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libeqtl_cuda.so")

EQTL_OK = 0
ERRORS = {-1: "EQTL_E_ARG", -2: "EQTL_E_CUDA", -3: "EQTL_E_NOMEM", -4: "EQTL_E_STATE", -5: "EQTL_E_DEVICE",
          -6: "EQTL_E_UNSUPPORTED", -7: "EQTL_E_OVERFLOW", -8: "EQTL_E_INTERNAL"}
MISS_FILTER, MISS_IMPUTE = 0, 1
PREC_SPLIT_F16, PREC_SPLIT_BF16, PREC_FP32_SIMT = 0, 1, 2

# every symbol include/eqtl_b200.h declares
EXPORTS = ["eqtl_open", "eqtl_close", "eqtl_last_error", "eqtl_set_precision", "eqtl_geno_load_bed",
           "eqtl_geno_dosage", "eqtl_scan_trans_lm", "eqtl_grm", "eqtl_lmm_basis", "eqtl_lmm_set_basis",
           "eqtl_scan_trans_lmm", "eqtl_stage_ms", "eqtl_launch_count", "eqtl_lmm_form", "eqtl_lmm_rotate",
           "eqtl_stream", "eqtl_pheno_load", "eqtl_t_tail", "eqtl_grm_noalloc", "eqtl_geno_dosage_rows",
           "eqtl_test_pairs", "eqtl_geno_load_dosage", "eqtl_scan_glm", "eqtl_pheno_int",
           "eqtl_peer", "eqtl_glm_mu", "eqtl_vcf_parse", "eqtl_lmm_basis_fast", "eqtl_pheno_permute",
           "eqtl_geno_subset"]
GRM_NOALLOC_MAX_N = 512
STAGES = {"decode": 0, "grm": 1, "eigen": 2, "rotate": 3, "prep": 4, "scan": 5, "refine": 6}


class GeneResult(C.Structure):
    _fields_ = [("n_tested", C.c_int32), ("acat_used", C.c_int32), ("acat_tan_sum", C.c_double),
                ("best_snp", C.c_int64), ("best_p", C.c_double), ("best_beta", C.c_double),
                ("best_se", C.c_double), ("best_t", C.c_double), ("best_r2", C.c_double)]


class Pair(C.Structure):
    _fields_ = [("snp", C.c_int64), ("gene", C.c_int32), ("reserved", C.c_int32), ("beta", C.c_double),
                ("se", C.c_double), ("t", C.c_double), ("p", C.c_double), ("r2", C.c_double)]


class ScanParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_genes", C.c_int32), ("p", C.c_int32), ("exclude_cis", C.c_int32),
                ("pthr", C.c_double), ("perm_thr", C.c_double),
                ("gene_chrom", C.POINTER(C.c_int32)), ("gene_lo", C.POINTER(C.c_int64)),
                ("gene_hi", C.POINTER(C.c_int64)), ("snp_chrom", C.POINTER(C.c_int32)),
                ("snp_pos", C.POINTER(C.c_int64)), ("y_rotated", C.c_int32)]


GENE_DTYPE = np.dtype([("n_tested", np.int32), ("acat_used", np.int32), ("acat_tan_sum", np.float64),
                       ("best_snp", np.int64), ("best_p", np.float64), ("best_beta", np.float64),
                       ("best_se", np.float64), ("best_t", np.float64), ("best_r2", np.float64)])
PAIR_DTYPE = np.dtype([("snp", np.int64), ("gene", np.int32), ("reserved", np.int32), ("beta", np.float64),
                       ("se", np.float64), ("t", np.float64), ("p", np.float64), ("r2", np.float64)])
assert GENE_DTYPE.itemsize == C.sizeof(GeneResult) and PAIR_DTYPE.itemsize == C.sizeof(Pair)

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built: run `python -m eqtl_b200.build`")
        lib = C.CDLL(LIB_PATH)
        vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        lib.eqtl_open.argtypes = [C.c_int, C.POINTER(vp)]
        lib.eqtl_close.argtypes = [vp]
        lib.eqtl_close.restype = None
        lib.eqtl_last_error.argtypes = [vp]
        lib.eqtl_last_error.restype = C.c_char_p
        lib.eqtl_set_precision.argtypes = [vp, C.c_int]
        lib.eqtl_geno_load_bed.argtypes = [vp, vp, i64, i64, i32, vp, i32, i32, dp, dp, vp, vp, vp,
                                           C.POINTER(i64)]
        lib.eqtl_geno_load_dosage.argtypes = [vp, vp, i64, i32, vp, i32, i32, dp, dp, vp, vp, vp, vp]
        lib.eqtl_geno_dosage.argtypes = [vp, i64, i64, vp]
        lib.eqtl_pheno_int.argtypes = [vp, vp, i32, i32]
        lib.eqtl_glm_mu.argtypes = [vp, vp]
        lib.eqtl_peer.argtypes = [vp, vp, i32, i32, i32, i32, dp, vp, vp, vp, C.POINTER(i32)]
        lib.eqtl_geno_dosage_rows.argtypes = [vp, vp, i64, vp]
        lib.eqtl_test_pairs.argtypes = [vp, i32, vp, vp, vp, vp, vp, i64, vp, vp]
        lib.eqtl_scan_trans_lm.argtypes = [vp, C.POINTER(ScanParams), vp, vp, vp, vp, i64, C.POINTER(i64), vp,
                                           i64, C.POINTER(i64)]
        lib.eqtl_grm.argtypes = [vp, vp, vp, C.POINTER(i64)]
        lib.eqtl_grm_noalloc.argtypes = [vp, vp, i64, i64, vp, i32, i32, dp, dp, vp, vp, C.POINTER(i64)]
        lib.eqtl_stage_ms.argtypes = [vp, C.c_int, C.POINTER(dp)]
        lib.eqtl_launch_count.argtypes = [vp, C.POINTER(C.c_uint64)]
        lib.eqtl_lmm_form.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        lib.eqtl_lmm_rotate.argtypes = [vp]
        lib.eqtl_stream.argtypes = [vp, C.POINTER(vp)]
        lib.eqtl_pheno_load.argtypes = [vp, vp, vp, i32, i32, i32]
        lib.eqtl_geno_subset.argtypes = [vp, vp, i32]
        lib.eqtl_pheno_permute.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32, C.c_uint64, vp, i32, vp]
        lib.eqtl_t_tail.argtypes = [vp, dp, vp, i64, i32, vp, vp, vp]
        lib.eqtl_lmm_basis.argtypes = [vp, vp, i32, vp, vp]
        lib.eqtl_lmm_set_basis.argtypes = [vp, vp, vp, i32]
        lib.eqtl_scan_trans_lmm.argtypes = [vp, C.POINTER(ScanParams), vp, vp, vp, vp, vp, i64, C.POINTER(i64),
                                            vp, i64, C.POINTER(i64)]
        lib.eqtl_scan_glm.argtypes = [vp, C.POINTER(ScanParams), vp, vp, vp, vp, vp, vp, i64, C.POINTER(i64),
                                      vp, i64, C.POINTER(i64)]
        _lib = lib
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class EqtlError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Context:
    """One device context (eqtl_open / eqtl_close)."""

    def __init__(self, device: int = 0, precision: int = PREC_SPLIT_F16):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.eqtl_open(device, C.byref(h))
        if rc != EQTL_OK:
            raise EqtlError(rc, "eqtl_open failed")
        self.h = h
        self.device = device
        if precision != PREC_SPLIT_F16:
            self._check(self.lib.eqtl_set_precision(self.h, precision))
        self.n_kept = 0
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.eqtl_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != EQTL_OK:
            raise EqtlError(rc, self.lib.eqtl_last_error(self.h).decode())

    # -- genotypes
    def load_bed(self, rows: np.ndarray, n_file: int, sample_col, miss_hand: int = MISS_IMPUTE,
                 max_miss: float = 0.8, maf_min: float = 0.0):
        rows = np.ascontiguousarray(rows, dtype=np.uint8)
        col = np.ascontiguousarray(sample_col, dtype=np.int32)
        m = rows.shape[0]
        keep = np.zeros(m, np.uint8)
        af = np.zeros(m, np.float64)
        nm = np.zeros(m, np.int32)
        nk = C.c_int64()
        self._check(self.lib.eqtl_geno_load_bed(self.h, _ptr(rows), m, rows.shape[1] if m else (n_file + 3) // 4,
                                                n_file, _ptr(col), col.size, miss_hand, max_miss, maf_min,
                                                _ptr(keep), _ptr(af), _ptr(nm), C.byref(nk)))
        self.n_kept = nk.value
        self.n = self.n_full = col.size
        return keep.astype(bool), af, nm

    def load_dosage(self, ds: np.ndarray, sample_col, miss_hand: int = MISS_IMPUTE, max_miss: float = 0.8,
                    maf_min: float = 0.0):
        """FP32 dosage rows [m, n_file] (NaN = missing call) instead of .bed rows."""
        ds = np.ascontiguousarray(ds, dtype=np.float32)
        col = np.ascontiguousarray(sample_col, dtype=np.int32)
        m, n_file = ds.shape
        keep = np.zeros(m, np.uint8)
        af = np.zeros(m, np.float64)
        nm = np.zeros(m, np.int32)
        nk = C.c_int64()
        self._check(self.lib.eqtl_geno_load_dosage(self.h, _ptr(ds), m, n_file, _ptr(col), col.size, miss_hand,
                                                   max_miss, maf_min, _ptr(keep), _ptr(af), _ptr(nm),
                                                   C.byref(nk)))
        self.n_kept = nk.value
        self.n = self.n_full = col.size
        return keep.astype(bool), af, nm

    def pheno_int(self, Y: np.ndarray) -> np.ndarray:
        """eqtl_pheno_int: the rank-based inverse normal transform of every column of Y [n, G]."""
        out = np.array(Y, dtype=np.float64, order="F", copy=True)
        self._check(self.lib.eqtl_pheno_int(self.h, _ptr(out), out.shape[0], out.shape[1]))
        return out

    def peer(self, Y: np.ndarray, k: int, max_iter: int, tol: float, X0: np.ndarray, W0: np.ndarray):
        """eqtl_peer: PEER factors of Y [n, G] from X0 [n, k], W0 [G, k] -> (X [n, k], iterations)."""
        Y = np.asfortranarray(Y, dtype=np.float64)
        X0 = np.asfortranarray(X0, dtype=np.float64)
        W0 = np.asfortranarray(W0, dtype=np.float64)
        n, G = Y.shape
        X = np.zeros((n, k), np.float64, order="F")
        it = C.c_int32()
        self._check(self.lib.eqtl_peer(self.h, _ptr(Y), n, G, k, max_iter, tol, _ptr(X0), _ptr(W0), _ptr(X),
                                       C.byref(it)))
        return X, it.value

    def geno_subset(self, idx=None):
        """eqtl_geno_subset: restrict the loaded genotypes to the analysis
        samples idx (increasing positions); None restores them all."""
        if idx is None:
            self._check(self.lib.eqtl_geno_subset(self.h, None, 0))
            self.n = self.n_full
            return
        idx = np.ascontiguousarray(idx, np.int32)
        self._check(self.lib.eqtl_geno_subset(self.h, _ptr(idx), idx.size))
        self.n = idx.size

    def dosage(self, lo: int, hi: int) -> np.ndarray:
        out = np.zeros((hi - lo, self.n), np.float64)
        self._check(self.lib.eqtl_geno_dosage(self.h, lo, hi, _ptr(out)))
        return out

    # -- scans
    @staticmethod
    def _params(n, G, p, pthr, perm_thr, windows):
        prm = ScanParams()
        prm.n, prm.n_genes, prm.p = n, G, p
        prm.pthr, prm.perm_thr = pthr, perm_thr
        keep = []
        if windows is not None:
            gchrom, glo, ghi, schrom, spos, exclude = windows
            arrs = [np.ascontiguousarray(gchrom, np.int32), np.ascontiguousarray(glo, np.int64),
                    np.ascontiguousarray(ghi, np.int64), np.ascontiguousarray(schrom, np.int32),
                    np.ascontiguousarray(spos, np.int64)]
            keep = arrs
            prm.gene_chrom = arrs[0].ctypes.data_as(C.POINTER(C.c_int32))
            prm.gene_lo = arrs[1].ctypes.data_as(C.POINTER(C.c_int64))
            prm.gene_hi = arrs[2].ctypes.data_as(C.POINTER(C.c_int64))
            prm.snp_chrom = arrs[3].ctypes.data_as(C.POINTER(C.c_int32))
            prm.snp_pos = arrs[4].ctypes.data_as(C.POINTER(C.c_int64))
            prm.exclude_cis = int(exclude)   # 0 gw, 1 trans (skip the window), 2 cis (only the window)
        return prm, keep

    def pheno_load(self, Y, X):
        """eqtl_pheno_load: keep Y [n, G] and X [n, p] resident on the device."""
        Y = np.asfortranarray(Y, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        self._check(self.lib.eqtl_pheno_load(self.h, _ptr(Y), _ptr(X), Y.shape[0], Y.shape[1], X.shape[1]))
        self.pheno_shape = (Y.shape[0], Y.shape[1], X.shape[1])

    def pheno_permute(self, base, X, gene_key, n_perm: int, seed: int, xb0=None, dinv=None, out: bool = False):
        """eqtl_pheno_permute: the resident phenotypes become n_perm device-drawn
        permutations of each gene's base vector (base, xb0, dinv [n, G]; LMM form
        when xb0 and dinv are given); returns the columns [n, G * n_perm] when
        out is True."""
        base = np.asfortranarray(base, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        n, G = base.shape
        if (xb0 is None) != (dinv is None):
            raise ValueError("give both xb0 and dinv, or neither")
        if xb0 is not None:
            xb0 = np.asfortranarray(xb0, dtype=np.float64)
            dinv = np.asfortranarray(dinv, dtype=np.float64)
            assert xb0.shape == base.shape and dinv.shape == base.shape
        keys = np.ascontiguousarray(gene_key, np.uint64)
        assert keys.size == G
        Y = np.zeros((n, G * n_perm), np.float64, order="F") if out else None
        self._check(self.lib.eqtl_pheno_permute(self.h, _ptr(base), _ptr(xb0), _ptr(dinv), _ptr(keys), n, G, n_perm,
                                                C.c_uint64(seed), _ptr(X), X.shape[1], _ptr(Y)))
        self.pheno_shape = (n, G * n_perm, X.shape[1])
        return Y

    def _scan(self, fn, Y, X, pthr, perm_thr, windows, extra=(), rotated=False):
        if Y is None:
            n, G, p = self.pheno_shape        # resident phenotypes
        else:
            Y = np.asfortranarray(Y, dtype=np.float64)   # [n, G] column-major
            X = np.asfortranarray(X, dtype=np.float64)   # [n, p]
            (n, G), p = Y.shape, X.shape[1]
        prm, keep = self._params(n, G, p, pthr, perm_thr, windows)
        prm.y_rotated = 1 if rotated else 0
        genes = np.zeros(G, GENE_DTYPE)
        cap = 1 << 16
        while True:
            pairs = np.zeros(cap, PAIR_DTYPE)
            cands = np.zeros(cap, PAIR_DTYPE)
            npair, ncand = C.c_int64(), C.c_int64()
            rc = fn(self.h, C.byref(prm), _ptr(Y), _ptr(X), *extra, _ptr(genes), _ptr(pairs), cap, C.byref(npair),
                    _ptr(cands), cap, C.byref(ncand))
            if rc == -7 and max(npair.value, ncand.value) > cap:
                cap = max(npair.value, ncand.value)
                continue
            self._check(rc)
            return genes, pairs[: npair.value], cands[: ncand.value]

    def scan_trans_lm(self, Y, X, pthr, perm_thr=0.0, windows=None):
        """eqtl_scan_trans_lm: Y [n, G] (gene columns), X [n, p] with intercept."""
        return self._scan(self.lib.eqtl_scan_trans_lm, Y, X, pthr, perm_thr, windows)

    def stage_ms(self, stage: str) -> float:
        """Device time of a pipeline stage in the last call that ran it."""
        v = C.c_double()
        self._check(self.lib.eqtl_stage_ms(self.h, STAGES[stage], C.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = C.c_uint64()
        self._check(self.lib.eqtl_launch_count(self.h, C.byref(v)))
        return v.value

    def lmm_form(self):
        """(node deltas, K columns per accumulator) of the most recent LMM
        scan's interpolated gg and a_k; (0, 0) for the direct form."""
        a, b = C.c_int32(), C.c_int32()
        self._check(self.lib.eqtl_lmm_form(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def t_tail(self, df: float, t, use_smem: bool = False, screen: bool = False):
        """Device Student-t tail -> (-log10 p, ACAT term, flags); with
        screen=True the scan epilogues' ACAT screen -> (|t|, term, flags)."""
        t = np.ascontiguousarray(t, np.float32)
        nl = np.zeros(t.size, np.float32)
        term = np.zeros(t.size, np.float64)
        fl = np.zeros(t.size, np.uint8)
        self._check(self.lib.eqtl_t_tail(self.h, df, _ptr(t), t.size, int(use_smem) | (2 if screen else 0), _ptr(nl),
                                         _ptr(term), _ptr(fl)))
        return nl, term, fl

    def stream_ptr(self) -> int:
        v = C.c_void_p()
        self._check(self.lib.eqtl_stream(self.h, C.byref(v)))
        return v.value or 0

    def rotate(self):
        self._check(self.lib.eqtl_lmm_rotate(self.h))

    def grm(self):
        """eqtl_grm -> (K [n, n], N_packed [n(n+1)/2], m_used)."""
        K = np.zeros((self.n, self.n), np.float64)
        N = np.zeros(self.n * (self.n + 1) // 2, np.int32)
        mu = C.c_int64()
        self._check(self.lib.eqtl_grm(self.h, _ptr(K), _ptr(N), C.byref(mu)))
        return K, N, mu.value

    def grm_noalloc(self, bed_dev: int, m: int, bytes_per_snp: int, col_dev: int, n: int, K_dev: int,
                    N_dev: int = 0, miss_hand: int = MISS_IMPUTE, max_miss: float = 0.8,
                    maf_min: float = 0.0) -> int:
        """eqtl_grm_noalloc on caller-owned device buffers (raw device
        pointers); returns the number of SNPs used."""
        mu = C.c_int64()
        self._check(self.lib.eqtl_grm_noalloc(self.h, C.c_void_p(bed_dev), m, bytes_per_snp, C.c_void_p(col_dev), n,
                                              miss_hand, max_miss, maf_min, C.c_void_p(K_dev),
                                              C.c_void_p(N_dev) if N_dev else None, C.byref(mu)))
        return mu.value

    def lmm_basis(self, K=None, outputs=True):
        """eqtl_lmm_basis -> (lambda [n], Q [n, n] with eigenvectors as columns);
        with outputs=False the basis only stays resident and None is returned."""
        n = self.n if K is None else K.shape[0]
        lam = np.zeros(n, np.float64) if outputs else None
        Qc = np.zeros(n * n, np.float64) if outputs else None
        Kc = None if K is None else np.ascontiguousarray(K, np.float64)
        self._check(self.lib.eqtl_lmm_basis(self.h, _ptr(Kc), n, _ptr(lam), _ptr(Qc)))
        return (lam, Qc.reshape(n, n).T) if outputs else None

    def set_basis(self, Q, lam):
        """eqtl_lmm_set_basis with Q [n, n] (eigenvectors as columns)."""
        Qc = np.ascontiguousarray(np.asarray(Q, np.float64).T)   # column-major
        lam = np.ascontiguousarray(lam, np.float64)
        self._check(self.lib.eqtl_lmm_set_basis(self.h, _ptr(Qc), _ptr(lam), lam.size))

    def test_pairs(self, model: str, Y, X, cols, snps):
        """eqtl_test_pairs: FP64 statistics of (column of Y, kept SNP) pairs
        -> (pairs [k] PAIR_DTYPE, delta [G] or None)."""
        Y = np.asfortranarray(Y, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        (n, G), p = Y.shape, X.shape[1]
        prm, _ = self._params(n, G, p, 0.0, 0.0, None)
        cols = np.ascontiguousarray(cols, np.int32)
        snps = np.ascontiguousarray(snps, np.int64)
        out = np.zeros(cols.size, PAIR_DTYPE)
        delta = np.zeros(G, np.float64) if model == "lmm" else None
        self._check(self.lib.eqtl_test_pairs(self.h, 0 if model == "lm" else 1, C.byref(prm), _ptr(Y), _ptr(X),
                                             _ptr(cols), _ptr(snps), cols.size, _ptr(out), _ptr(delta)))
        return out, delta

    def scan_glm(self, Y, X, pthr, perm_thr=0.0, windows=None):
        """eqtl_scan_glm -> (genes, pairs, cands, phi, converged); pairs' t is the score z."""
        G = self.pheno_shape[1] if Y is None else np.asarray(Y).shape[1]
        phi = np.zeros(G, np.float64)
        conv = np.zeros(G, np.uint8)
        genes, pairs, cands = self._scan(self.lib.eqtl_scan_glm, Y, X, pthr, perm_thr, windows,
                                         extra=(_ptr(phi), _ptr(conv)))
        return genes, pairs, cands, phi, conv.astype(bool)

    def scan_trans_lmm(self, Y, X, pthr, perm_thr=0.0, windows=None, rotated=False):
        """eqtl_scan_trans_lmm -> (genes, pairs, cands, delta); rotated: the
        columns are already in the eigenbasis (y_rotated)."""
        delta = np.zeros(self.pheno_shape[1] if Y is None else np.asarray(Y).shape[1], np.float64)
        genes, pairs, cands = self._scan(self.lib.eqtl_scan_trans_lmm, Y, X, pthr, perm_thr, windows,
                                         extra=(_ptr(delta),), rotated=rotated)
        return genes, pairs, cands, delta
