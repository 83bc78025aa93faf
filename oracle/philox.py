"""CPU restatement of the device-drawn permutations (numpy).

TEST INFRASTRUCTURE ONLY: the checker of eqtl_pheno_permute; the product
never imports it.

The reference draws gene-level permutations with std::mt19937 and
std::shuffle (include/eqtl/scan_cis.hpp:102-147, src/scan_perm.cpp:80-132);
the host program reproduces those sequences exactly. The device mode draws
them from a counter-based generator instead, so this module restates that
mode's definition, not the reference:

* Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
  as easy as 1, 2, 3", SC 2011): ten rounds of
      (c0, c1, c2, c3) -> (hi(M1 c2) ^ c1 ^ k0, lo(M1 c2), hi(M0 c0) ^ c3 ^ k1, lo(M0 c0))
  with M0 = 0xD2511F53, M1 = 0xCD9E8D57, the key bumped by (0x9E3779B9,
  0xBB67AE85) between rounds. Pinned by the published known-answer vectors
  (tests/test_philox.py).
* Permutation b of gene g over n samples: sample i gets the 32-bit word
  i % 4 of Philox(counter = (b, i // 4, lo32(gene_key), hi32(gene_key)),
  key = (lo32(seed), hi32(seed))); the permutation lists the samples in
  increasing order of their words, ties in increasing sample order.
* The gene key is the 64-bit FNV-1a hash of the gene name.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, key) -> np.ndarray:
    """ctr [N, 4] uint32 counters, key (k0, k1) -> [N, 4] uint32 words."""
    c = np.asarray(ctr, np.uint64).copy()
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c[:, 0]
        p1 = M1 * c[:, 2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = np.stack([hi1 ^ c[:, 1] ^ np.uint64(k0), lo1, hi0 ^ c[:, 3] ^ np.uint64(k1), lo0], axis=1)
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c.astype(np.uint32)


def fnv1a64(name: str) -> int:
    h = 0xCBF29CE484222325
    for b in name.encode():
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def permutation(n: int, b: int, gene_key: int, seed: int) -> np.ndarray:
    """Sample order of permutation b of the gene with key gene_key."""
    q = (n + 3) // 4
    ctr = np.zeros((q, 4), np.uint64)
    ctr[:, 0] = b
    ctr[:, 1] = np.arange(q)
    ctr[:, 2] = gene_key & 0xFFFFFFFF
    ctr[:, 3] = gene_key >> 32
    words = philox4x32_10(ctr, (seed & 0xFFFFFFFF, seed >> 32)).reshape(-1)[:n]
    return np.argsort(words, kind="stable")


def permuted_columns(base: np.ndarray, gene_keys, n_perm: int, seed: int, xb0=None, dinv=None) -> np.ndarray:
    """The columns eqtl_pheno_permute makes: base, xb0, dinv [n, G] ->
    [n, G * n_perm], column g * n_perm + b."""
    n, G = base.shape
    out = np.empty((n, G * n_perm))
    for g in range(G):
        for b in range(n_perm):
            v = base[permutation(n, b, int(gene_keys[g]), seed), g]
            if xb0 is not None:
                v = xb0[:, g] + v / np.sqrt(np.maximum(dinv[:, g], 1e-12))
            out[:, g * n_perm + b] = v
    return out
