"""The GPU sieve and its scans through the C ABI, bit-exact against the oracle on seeded
ranges, against the reference's golden pi / twin / sextuplet windows, and against the
full-size fixtures (tests/golden/configs.json)."""
import numpy as np
import pytest

from helpers import brute_range

pytestmark = pytest.mark.gpu

KEYS = ("pi", "twins", "max_gap", "gap_start", "tuple6", "tuple6_cks", "first_prime", "last_prime")


def same(a, b):
    return all(int(a[k]) == int(b[k]) for k in KEYS)


@pytest.mark.parametrize("lo,hi", [(0, 300), (1, 3), (2, 3), (3, 4), (0, 2), (4, 5), (7, 200), (8, 97), (97, 98),
                                   (1000, 1100), (1001, 1099), (99990, 100120), (0, 10 ** 6)])
def test_tiny_ranges_brute(engine, lo, hi):
    r = engine.sieve_range(lo, hi, hash_log2=4, bitmap=True)
    b = brute_range(lo, hi, hash_log2=4)
    for k in ("pi", "twins", "tuple6", "first_prime", "last_prime", "max_gap", "gap_start"):
        assert r[k] == b[k], (k, r[k], b[k])
    bits = np.unpackbits(r["bitmap"].view(np.uint8), bitorder="little")[: len(b["bits"])]
    assert np.array_equal(bits, b["bits"])
    assert [int(x) for x in r["hashes"]] == b["hashes"]


def ranges(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        h = int(10 ** rng.uniform(0, 13))
        L = int(2 ** rng.uniform(0, 24))
        out.append((h, h + max(L, 1)))
    return out


@pytest.mark.parametrize("tile", [18, 19, 20])
def test_random_ranges_vs_oracle(engine, orc, tile):
    for lo, hi in ranges(100 + tile, 40):
        r = engine.sieve_range(lo, hi, tile_log2=tile, hash_log2=12, bitmap=True)
        o = orc.sieve_range(lo, hi, hash_log2=12, bitmap=True)
        assert same(r, o), (lo, hi, {k: (r[k], o[k]) for k in KEYS})
        assert np.array_equal(r["bitmap"], o["bitmap"]), (lo, hi)
        assert np.array_equal(r["hashes"], o["hashes"]), (lo, hi)


@pytest.mark.parametrize("lo", [10 ** 15, 10 ** 17 + 12345, 2 ** 62 + 1, 10 ** 18, 2 ** 64 - 2 ** 26])
def test_high_ranges_vs_oracle(engine, orc, lo):
    hi = lo + 3 * 2 ** 21 + 12345
    if hi > 2 ** 64 - 2 ** 18:
        hi = 2 ** 64 - 2 ** 18
    r = engine.sieve_range(lo, hi, block_log2=21, hash_log2=16)
    o = orc.sieve_range(lo, hi, block_log2=21, hash_log2=16)
    assert same(r, o), (lo, hi)
    assert np.array_equal(r["blocks"], o["blocks"])
    assert np.array_equal(r["hashes"], o["hashes"])


def test_plain_equals_batched(engine):
    import mathpub_b200 as mp
    for lo, hi in [(10 ** 15, 10 ** 15 + 2 ** 26), (10 ** 9 + 1, 10 ** 9 + 10 ** 7 + 1), (0, 2 ** 22)]:
        a = engine.sieve_range(lo, hi, block_log2=22, hash_log2=19, mode=mp.MODE_BATCHED)
        b = engine.sieve_range(lo, hi, block_log2=22, hash_log2=19, mode=mp.MODE_PLAIN)
        assert same(a, b)
        assert np.array_equal(a["blocks"], b["blocks"]) and np.array_equal(a["hashes"], b["hashes"])


def test_reference_pi_windows(engine, ref_vectors):
    for k in range(6, 13):
        assert engine.sieve_range(0, 10 ** k)["pi"] == ref_vectors["pi10"][str(k)], k
    for w in ref_vectors["pi_windows"]:
        assert engine.sieve_range(w["lo"], w["hi"])["pi"] == w["pi"], w


def test_reference_twin_counts(engine, ref_vectors):
    tw = ref_vectors["twins_below_10n"]
    for n in range(1, 13):
        assert engine.sieve_range(0, 10 ** n)["twins"] == tw[n - 1], n


def test_reference_sextuplet_windows(engine, ref_vectors, verify_py):
    # [1e15, 1e15 + 2e12) of A350826/a350826.c:2571 (verify_a350826.py's window)
    w = ref_vectors["sext_windows"][0]
    assert (w["lo"], w["hi"]) == ("1e15", "1e15+2e12")
    r = engine.sieve_range(10 ** 15, 10 ** 15 + 2 * 10 ** 12)
    assert (r["tuple6"], r["tuple6_cks"]) == (w["count"], w["cks"])
    a = ref_vectors["A350826"]
    for n in range(1, 13):
        r = engine.sieve_range(10 ** (n - 1), 10 ** n)
        assert r["tuple6"] == a[n], n
    for s in verify_py["sext"]:
        lo = int(float(s["lo"]))
        parts = s["hi"].split("+")
        hi = int(float(parts[0])) + (int(float(parts[1])) if len(parts) > 1 else 0)
        r = engine.sieve_range(lo, hi)
        assert (r["tuple6"], r["tuple6_cks"]) == (s["count"], s["cks"])


def test_config1_fixture(engine, configs):
    c = configs["config1"]
    r = engine.sieve_range(c["lo"], c["hi"], hash_log2=c["hash_log2"])
    assert {k: r[k] for k in KEYS} == c["stats"]
    assert [int(x) for x in r["hashes"]] == c["hashes"]


def test_config2_fixture(engine, configs):
    """[1e15, 1e15 + 2^34): per-2^24 block stats, 2^20-integer segment hashes, range stats."""
    import oracle
    c = configs["config2"]
    r = engine.sieve_range(c["lo"], c["hi"], block_log2=c["block_log2"], hash_log2=c["hash_log2"])
    assert {k: r[k] for k in KEYS} == c["stats"]
    bl = r["blocks"]
    assert len(bl) == c["nblocks"]
    arr = np.ascontiguousarray(np.stack([bl[n] for n in bl.dtype.names], axis=1).reshape(-1))
    assert int(oracle.o().or_fnv1a64(arr.ctypes.data, arr.nbytes)) == c["blocks_fnv"]
    h = np.ascontiguousarray(r["hashes"])
    assert len(h) == c["nhashes"]
    assert int(oracle.o().or_fnv1a64(h.ctypes.data, h.nbytes)) == c["hashes_fnv"]
    # size-independent properties: blocks add up to the range, maximal gap is a block maximum
    assert int(bl["pi"].sum()) == r["pi"] and int(bl["tuple6"].sum()) == r["tuple6"]
    assert int(bl["max_gap"].max()) == r["max_gap"]


def test_primes_range(engine, orc):
    for lo, hi in [(0, 100000), (10 ** 12, 10 ** 12 + 10 ** 6), (2, 3), (5, 5 + 1)]:
        assert np.array_equal(engine.primes_range(lo, hi), orc.primes_range(lo, hi))


def test_errors_are_reported(engine):
    import mathpub_b200 as mp
    with pytest.raises(mp.MathpubError):
        engine.sieve_range(10, 5)
    with pytest.raises(mp.MathpubError):
        engine.sieve_range(2 ** 64 - 2, 2 ** 64 - 1)
    with pytest.raises(mp.MathpubError):
        engine.sieve_range(0, 100, tile_log2=17)
    # the handle still works afterwards
    assert engine.sieve_range(0, 100)["pi"] == 25


def test_graph_replay_after_buffer_growth(engine):
    """A batched call is captured as a CUDA graph and replayed when it repeats; a larger call in
    between reallocates the scratch buffers, which must retire the older graph."""
    a = (10 ** 12, 10 ** 12 + 2 ** 24)
    first = engine.sieve_range(*a, block_log2=22, hash_log2=18)
    engine.sieve_range(10 ** 13, 10 ** 13 + 2 ** 33, block_log2=24, hash_log2=22)
    for _ in range(3):
        again = engine.sieve_range(*a, block_log2=22, hash_log2=18)
        assert same(first, again)
        assert np.array_equal(first["blocks"], again["blocks"]) and np.array_equal(first["hashes"], again["hashes"])
