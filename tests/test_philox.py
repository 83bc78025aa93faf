"""The device permutation mode's definition, restated on the CPU (oracle/philox.py):
Philox4x32-10 against the known-answer vectors published with the algorithm
(Salmon et al., SC 2011; the Random123 distribution's kat_vectors), FNV-1a
64 against its published test values, and the permutation construction's
uniformity. The -m gpu test (test_gpu_perm_device.py) checks the device
against this restatement bit for bit."""
import itertools
import math
import os
import subprocess
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import philox  # noqa: E402

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "eqtl_b200", "bin", "eqtl")

KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    got = philox.philox4x32_10(np.array([ctr], np.uint64), key)[0]
    assert [int(x) for x in got] == list(want)


def test_fnv1a64_test_values():
    assert philox.fnv1a64("") == 0xCBF29CE484222325
    assert philox.fnv1a64("a") == 0xAF63DC4C8601EC8C
    assert philox.fnv1a64("foobar") == 0x85944171F73967E8


def test_permutations_are_uniform():
    """n = 4: the 24 orders over 4,800 draws (two genes), chi-square at 1e-4."""
    n, B = 4, 2400
    counts = {p: 0 for p in itertools.permutations(range(n))}
    for key in (philox.fnv1a64("G1"), philox.fnv1a64("G2")):
        for b in range(B):
            counts[tuple(int(i) for i in philox.permutation(n, b, key, 7))] += 1
    e = 2 * B / 24
    chi2 = sum((c - e) ** 2 / e for c in counts.values())
    assert chi2 < 60.0, chi2  # 23 degrees of freedom: P(chi2 > 60) ~ 3e-5


def test_position_frequencies_are_uniform():
    """n = 50, 2,000 draws: where sample 0 lands, chi-square over 50 slots."""
    n, B = 50, 2000
    key = philox.fnv1a64("ENSG00000000003")
    where = np.zeros(n)
    for b in range(B):
        where[int(np.nonzero(philox.permutation(n, b, key, 1) == 0)[0][0])] += 1
    e = B / n
    chi2 = float(((where - e) ** 2 / e).sum())
    assert chi2 < 100.0, chi2  # 49 degrees of freedom: P(chi2 > 100) ~ 2e-5


def test_columns_lm_and_lmm_forms():
    rng = np.random.default_rng(3)
    n, G, B = 9, 3, 4
    base = rng.normal(size=(n, G))
    xb0 = rng.normal(size=(n, G))
    dinv = rng.uniform(0.1, 2.0, size=(n, G))
    keys = [philox.fnv1a64(f"g{g}") for g in range(G)]
    lm = philox.permuted_columns(base, keys, B, 5)
    lmm = philox.permuted_columns(base, keys, B, 5, xb0, dinv)
    for g in range(G):
        for b in range(B):
            c = g * B + b
            assert sorted(lm[:, c]) == sorted(base[:, g])
            perm = philox.permutation(n, b, keys[g], 5)
            np.testing.assert_array_equal(lmm[:, c], xb0[:, g] + base[perm, g] / np.sqrt(dinv[:, g]))
    # seeds and permutation indices give different draws
    assert not np.array_equal(lm, philox.permuted_columns(base, keys, B, 6))
    assert len({tuple(philox.permutation(n, b, keys[0], 5)) for b in range(B)}) == B


@pytest.mark.skipif(not os.path.exists(BIN), reason="host program not built")
def test_cli_rejects_unknown_perm_rng():
    r = subprocess.run([BIN, "-b", "x", "-e", "y", "--perm-rng", "fast"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode != 0 and "--perm-rng" in r.stderr
    h = subprocess.run([BIN, "--help"], capture_output=True, text=True, timeout=60)
    assert "--perm-rng" in h.stdout + h.stderr
