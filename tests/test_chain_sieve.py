"""The constellation sieve (mp_chain_sieve): chains of consecutive primes with gaps 2, 4, 6, ...
(A016045) and with gaps ..., 6, 4, 2 (A263049), found from residue classes, rotated bit
patterns and base-2 screening without enumerating primes.

CPU: the oracle's restatement of decreasing chains (oracle.dec_chains, the walk of
gapchain/gapchain_ps.c:365-395) gives the reference's A263049 terms a(2..10).
GPU: increasing chains equal the enumeration (mp_gap_chains, itself pinned to the reference's
gapchain_ps and the oracle) head for head and length for length; decreasing chains equal the
oracle and the decreasing chains that the reference's own gapsieve program prints; both shapes
give the reference's terms, up to the records A016045 a(15) and A263049 a(15)."""
import os
import subprocess
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GAPSIEVE_CPU = os.path.join(ROOT, "oracle", "_ref", "gapsieve_cpu")


def dec_keys(heads, lens, k):
    """The start of the exact k-prime pattern in each decreasing chain (its last k primes)."""
    h = heads.astype(object)
    n = lens.astype(object)
    j = n - k
    return [int(a + b * (2 * c - 1 - b)) for a, b, c in zip(h, j, n)]


# ---- CPU: the oracle pinned ----

def test_oracle_dec_chains_give_a263049(orc, ref_vectors):
    a = ref_vectors["A263049"]
    for n in range(2, 9):                               # a(n): the first (n + 1)-prime pattern
        heads, lens, keys = orc.dec_chains(0, 4 * 10 ** 7, n + 1)
        assert int(keys.min()) == a[n - 1]
        assert dec_keys(heads, lens, n + 1) == [int(x) for x in keys]
    # a(9) starts the 10-prime pattern at the end of the 11-prime chain from a(10)
    heads, lens, keys = orc.dec_chains(245 * 10 ** 6, 246 * 10 ** 6, 10)
    assert [(int(h), int(l), int(k)) for h, l, k in zip(heads, lens, keys)] == [(a[9], 11, a[8])]


# ---- GPU: increasing chains ----

@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi,k", [
    (0, 10 ** 9, 4),                                    # the exact strip below 1024, then the sieve
    (0, 2 * 10 ** 8, 2),                                # short chains: the enumeration
    (2 ** 24 - 10 ** 6, 2 ** 24 + 10 ** 9, 4),
    (10 ** 12, 10 ** 12 + 10 ** 11, 5),
    (10 ** 12 + 7, 10 ** 12 + 3 * 10 ** 11 + 1, 6),
    (10 ** 15, 10 ** 15 + 2 * 10 ** 12, 8),
    (2 ** 62 - 10 ** 12, 2 ** 62, 7),
    (2 ** 64 - 2 ** 40, 2 ** 64 - 2 ** 18 - 2 ** 17, 5),   # the top of the enumeration's range
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


@pytest.mark.gpu
def test_constellation_sieve_finds_a016045(engine, ref_vectors):
    a = ref_vectors["A016045"]
    heads, lens = engine.chain_sieve(0, 10 ** 7, 4)
    assert [int(heads[np.argmax(lens >= L)]) for L in range(4, 8)] == a[2:6]
    heads, lens = engine.chain_sieve(0, 47 * 10 ** 11, 7)
    assert [int(heads[np.argmax(lens >= L)]) for L in range(7, 13)] == a[5:11]
    t0 = time.perf_counter()
    heads, lens = engine.chain_sieve(10 ** 14, 5 * 10 ** 14, 13)
    print(f"k=13 over [1e14, 5e14): {len(heads)} heads in {time.perf_counter() - t0:.2f} s")
    assert int(heads[np.argmax(lens >= 13)]) == a[11]       # a(12), a chain of 13 primes
    assert int(heads[np.argmax(lens >= 14)]) == a[12]       # a(13), 14 primes


@pytest.mark.gpu
@pytest.mark.parametrize("n,half", [(14, 4 * 10 ** 12), (15, 10 ** 13)])
def test_constellation_sieve_finds_a016045_record_heads(engine, ref_vectors, n, half):
    """a(14) = 221860944705726407 (15 primes) and a(15) = 1397398433200922807 (16 primes, gaps 2,
    4, ..., 30; the next gap is 60), the reference's gapsieve results: a window around each holds
    it as the first chain of n + 1 primes."""
    a = ref_vectors["A016045"][n - 1]
    t0 = time.perf_counter()
    heads, lens = engine.chain_sieve(a - half, a + half, n + 1)
    dt = time.perf_counter() - t0
    print(f"k={n + 1} over {2 * half:.3g} integers at {a:.4g}: {len(heads)} heads in {dt:.3f} s, "
          f"{2 * half / dt:.3g} integers/s")
    assert len(heads) >= 1 and int(heads[0]) == a
    if n == 15:
        assert int(lens[0]) == 16


# ---- GPU: decreasing chains ----

@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi,k", [
    (0, 10 ** 8, 4), (0, 10 ** 8, 6), (10 ** 9 - 10 ** 6, 10 ** 9 + 10 ** 8, 5),
    (10 ** 12, 10 ** 12 + 10 ** 10, 5), (2 ** 62 - 10 ** 10, 2 ** 62, 5), (245 * 10 ** 6, 246 * 10 ** 6, 10),
])
def test_decreasing_chains_match_oracle(engine, orc, lo, hi, k):
    gh, gl = engine.chain_sieve(lo, hi, k, dec=True)
    oh, ol, _ = orc.dec_chains(lo, hi, k)
    assert len(oh) > 0
    assert np.array_equal(gh, oh) and np.array_equal(gl, ol)


@pytest.mark.gpu
def test_decreasing_chains_give_a263049(engine, ref_vectors):
    a = ref_vectors["A263049"]
    for n, top in [(3, 10 ** 4), (5, 10 ** 6), (8, 10 ** 8), (9, 3 * 10 ** 8), (10, 3 * 10 ** 8),
                   (11, 3 * 10 ** 10), (12, 2 * 10 ** 14), (13, 31 * 10 ** 14)]:
        heads, lens = engine.chain_sieve(0, top, n + 1, dec=True)
        assert min(dec_keys(heads, lens, n + 1)) == a[n - 1], n
    # the records: a(15) = 253253149671986953 heads a 16-prime chain, and a(14) = a(15) + 30
    # is the 15-prime pattern at its end
    heads, lens = engine.chain_sieve(a[14] - 10 ** 13, a[14] + 10 ** 13, 16, dec=True)
    assert [(int(h), int(l)) for h, l in zip(heads, lens)][:1] == [(a[14], 16)]
    heads, lens = engine.chain_sieve(a[13] - 10 ** 12, a[13] + 10 ** 12, 15, dec=True)
    assert min(dec_keys(heads, lens, 15)) == a[13]
    assert (a[14], 16) in [(int(h), int(l)) for h, l in zip(heads, lens)]


def reference_chains(args):
    """(shape, first prime, length) of every chain the reference's gapsieve prints."""
    if not os.path.exists(GAPSIEVE_CPU):
        pytest.skip("oracle/_ref/gapsieve_cpu is not built")
    r = subprocess.run([GAPSIEVE_CPU, *args.split(), "-q"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-400:]
    out = set()
    for line in r.stdout.splitlines():
        tag, rest = (line[:3], line[4:]) if line[:3] in ("inc", "dec") else ("inc", line)
        n, members = rest.split(":", 1)
        out.add((tag, int(members.split()[0]), int(n)))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi,k", [(10 ** 12, 10 ** 12 + 10 ** 11, 7), (10 ** 15, 10 ** 15 + 10 ** 13, 9)])
def test_both_shapes_match_the_reference_program(engine, lo, hi, k):
    want = reference_chains(f"-l {k} -g both -s {lo} -e {hi - 1}")
    got = set()
    for tag, dec in (("inc", False), ("dec", True)):
        heads, lens = engine.chain_sieve(lo, hi, k, dec=dec)
        got |= {(tag, int(h), int(n)) for h, n in zip(heads, lens)}
    assert len(want) > 0 and got == want


# ---- GPU: the first chain (gapsieve --first) ----

@pytest.mark.gpu
def test_chain_first_finds_the_terms(engine, ref_vectors):
    a, d = ref_vectors["A016045"], ref_vectors["A263049"]
    assert engine.chain_first(0, 2 ** 63, 13) == (a[11], a[11], 13)           # A016045 a(12)
    assert engine.chain_first(0, 2 ** 63, 11, dec=True) == (d[9], d[9], 11)   # A263049 a(10)
    assert engine.chain_first(0, 2 ** 63, 10, dec=True) == (d[8], d[9], 11)   # a(9): the end of that chain
    # the records, from 1e16 below them
    assert engine.chain_first(a[14] - 10 ** 16, 2 ** 63, 16) == (a[14], a[14], 16)
    assert engine.chain_first(d[13] - 10 ** 16, 2 ** 63, 15, dec=True) == (d[13], d[14], 16)
    assert engine.chain_first(10 ** 12, 10 ** 12 + 10 ** 9, 20) is None


# ---- GPU: above 2^64, to the reference's ceiling ----

@pytest.mark.gpu
def test_chain_first128_finds_the_records_above_2_64(engine, ref_vectors):
    """A016045 a(16) = 254345176718302423991 (17 primes) and a(17) = 307223174679659356577 (18
    primes), A263049 a(16) = 134491669675212201371 (17 primes): the reference's newest terms."""
    a, d = ref_vectors["A016045"], ref_vectors["A263049"]
    top = 33 * 10 ** 23
    for term, k, dec in [(a[15], 17, False), (a[16], 18, False), (d[15], 17, True)]:
        t0 = time.perf_counter()
        r = engine.chain_first128(term - 10 ** 16, top, k, dec=dec)
        print(f"k={k} dec={dec}: {r} in {time.perf_counter() - t0:.2f} s")
        assert r == (term, term, k)


@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi,k", [(2 ** 64 - 5 * 10 ** 12, 2 ** 64 + 5 * 10 ** 12, 10),
                                     (10 ** 20, 10 ** 20 + 10 ** 13, 10)])
def test_chain_sieve128_matches_the_reference_program(engine, lo, hi, k):
    want = reference_chains(f"-l {k} -g both -s {lo} -e {hi - 1}")
    got = set()
    for tag, dec in (("inc", False), ("dec", True)):
        got |= {(tag, h, n) for h, n in engine.chain_sieve128(lo, hi, k, dec=dec)}
    assert len(want) > 0 and got == want


@pytest.mark.gpu
def test_chain_sieve128_equals_the_64_bit_call(engine):
    lo, hi = 10 ** 15, 10 ** 15 + 2 * 10 ** 12
    for dec in (False, True):
        h, n = engine.chain_sieve(lo, hi, 8, dec=dec)
        assert engine.chain_sieve128(lo, hi, 8, dec=dec) == [(int(x), int(y)) for x, y in zip(h, n)]
