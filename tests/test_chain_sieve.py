"""The constellation sieve (mp_chain_sieve): the heads of chains of consecutive primes with gaps
2, 4, 6, ... found from residue classes, rotated bit patterns and base-2 screening, without
enumerating primes, must equal the enumeration (mp_gap_chains, itself checked against the
reference's gapchain_ps and the oracle) head for head and length for length, and give the
reference's A016045 terms."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lo,hi,k", [
    (2 ** 24 - 10 ** 6, 2 ** 24 + 10 ** 9, 4),          # across the enumerated low part
    (10 ** 12, 10 ** 12 + 10 ** 11, 5),
    (10 ** 12 + 7, 10 ** 12 + 3 * 10 ** 11 + 1, 6),
    (10 ** 15, 10 ** 15 + 2 * 10 ** 12, 8),
    (2 ** 62 - 10 ** 12, 2 ** 62, 7),
])
def test_constellation_sieve_equals_enumeration(engine, lo, hi, k):
    t0 = time.perf_counter()
    sh, sl = engine.chain_sieve(lo, hi, k)
    t1 = time.perf_counter()
    eh, el = engine.gap_chains(lo, hi, k)
    t2 = time.perf_counter()
    print(f"k={k} [{lo}, {hi}): {len(sh)} heads; sieve {t1 - t0:.3f} s, enumeration {t2 - t1:.3f} s")
    assert len(sh) > 0
    assert np.array_equal(sh, eh) and np.array_equal(sl, el)


def test_constellation_sieve_finds_a016045(engine, ref_vectors):
    a = ref_vectors["A016045"]
    heads, lens = engine.chain_sieve(0, 47 * 10 ** 11, 7)
    assert [int(heads[np.argmax(lens >= L)]) for L in range(7, 13)] == a[5:11]
    t0 = time.perf_counter()
    heads, lens = engine.chain_sieve(10 ** 14, 5 * 10 ** 14, 13)
    print(f"k=13 over [1e14, 5e14): {len(heads)} heads in {time.perf_counter() - t0:.2f} s")
    assert int(heads[np.argmax(lens >= 13)]) == a[11]       # a(12), a chain of 13 primes
    assert int(heads[np.argmax(lens >= 14)]) == a[12]       # a(13), 14 primes
