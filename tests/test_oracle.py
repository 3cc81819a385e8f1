"""The oracle (CPU restatement in oracle/mp_oracle.c) against the reference's own known
answers (tests/golden/ref_vectors.json, extracted from the reference's sources), against the
reference's Python verifiers (verify_py.json) and, where it was built, against the
reference's compiled C (oracle/_ref).  Runs on the CPU."""
import numpy as np
import pytest

from helpers import brute_range, fnv1a64, is_prime_td, mix64, tuple6_cks


def test_pseudoprime_lists(orc, ref_vectors):
    o = orc.o()
    # base-2 strong pseudoprimes (A350826/a350826.c:2467-2469): pass base 2, fail BPSW
    for n in ref_vectors["spsp2"]:
        assert o.or_sprp2(n) == 1 and o.or_slprp(n) == 0 and o.or_bpsw(n) == 0, n
    # strong Lucas pseudoprimes (:2477-2479): pass Lucas, fail base 2
    for n in ref_vectors["slpsp"]:
        assert o.or_slprp(n) == 1 and o.or_sprp2(n) == 0 and o.or_bpsw(n) == 0, n
    assert len(ref_vectors["spsp2"]) == 32 and len(ref_vectors["slpsp"]) == 32


def test_bpsw_against_reference_primality(orc):
    o = orc.o()
    for n in range(0, 20000):
        assert o.or_bpsw(n) == o.or_is_prime_ref(n) == is_prime_td(n), n
    rng = np.random.default_rng(7)
    xs = rng.integers(0, 2 ** 63, size=20000, dtype=np.uint64) * 2 + 1
    v = orc.bpsw(xs)
    ref = np.array([o.or_is_prime_ref(int(x)) for x in xs], dtype=bool)
    assert np.array_equal(v, ref)
    near = [2 ** 64 - 1 - 2 * k for k in range(300)]
    assert [o.or_bpsw(n) for n in near] == [o.or_is_prime_ref(n) for n in near]


def test_pi_and_twins_tables(orc, ref_vectors):
    # pi(10^k) of A158939/cuda/a158939_cuda.cu and pi(1e9) of A001220/wieferich.c; twin counts
    # below 10^n of A007508/README.md
    assert ref_vectors["pi_1e9"] == 50847534
    for k in range(6, 10):
        r = orc.sieve_range(0, 10 ** k)
        assert r["pi"] == ref_vectors["pi10"][str(k)]
        assert r["twins"] == ref_vectors["twins_below_10n"][k - 1]
    assert orc.sieve_range(0, 10 ** 9)["pi"] == ref_vectors["pi_1e9"]
    for n in range(1, 6):
        assert orc.sieve_range(0, 10 ** n)["twins"] == ref_vectors["twins_below_10n"][n - 1]


def test_pi_window_odd_bounds(orc, ref_vectors):
    w = [x for x in ref_vectors["pi_windows"] if x["lo"] == 12345000000][0]
    assert orc.sieve_range(w["lo"], w["hi"])["pi"] == w["pi"] == 42962974


def test_sextuplets_A350826(orc, ref_vectors):
    a = ref_vectors["A350826"]
    for n in range(1, 10):
        r = orc.sieve_range(10 ** (n - 1), 10 ** n)
        assert r["tuple6"] == a[n], n


def test_sextuplet_windows_verify_py(orc, verify_py):
    for w in verify_py["sext"]:
        lo, hi = int(float(w["lo"].split("+")[0])), None
        parts = w["hi"].split("+")
        hi = int(float(parts[0])) + (int(float(parts[1])) if len(parts) > 1 else 0)
        lo = int(float(w["lo"]))
        if hi - lo > 5 * 10 ** 9:
            continue
        r = orc.sieve_range(lo, hi)
        assert (r["tuple6"], r["tuple6_cks"]) == (w["count"], w["cks"]), w


def test_wieferich_windows_verify_py(orc, verify_py, ref_vectors):
    for w in verify_py["wieferich_base2"]:
        r = orc.wieferich_range(w["lo"], w["hi"])
        assert (r["primes"], r["cks"]) == (w["primes"], w["cks"]), w
        assert r["flt"] == 0
    r = orc.wieferich_range(1000, 4000)
    assert r["hits"] == ref_vectors["wieferich_base2"] == [1093, 3511]


@pytest.mark.parametrize("lo,hi", [(0, 300), (1, 3), (2, 3), (3, 4), (0, 2), (4, 5), (7, 200), (8, 97), (97, 98),
                                   (1000, 1100), (1001, 1099), (99990, 100120), (2 ** 20 - 100, 2 ** 20 + 300)])
def test_sieve_definitions_tiny(orc, lo, hi):
    r = orc.sieve_range(lo, hi, hash_log2=4, bitmap=True, nthreads=1)
    b = brute_range(lo, hi, hash_log2=4)
    for k in ("pi", "twins", "tuple6", "first_prime", "last_prime", "max_gap", "gap_start"):
        assert r[k] == b[k], (k, r[k], b[k])
    assert r["tuple6_cks"] == tuple6_cks(lo, hi)
    bits = np.unpackbits(r["bitmap"].view(np.uint8), bitorder="little")[: len(b["bits"])]
    assert np.array_equal(bits, b["bits"])
    assert [int(x) for x in r["hashes"]] == b["hashes"]


def test_blocks_sum_to_range(orc):
    lo, hi = 10 ** 12 + 12345, 10 ** 12 + 12345 + 3 * 2 ** 20 + 777
    r = orc.sieve_range(lo, hi, block_log2=20)
    bl = r["blocks"]
    assert int(bl["pi"].sum()) == r["pi"] and int(bl["twins"].sum()) == r["twins"]
    assert max(int(x) for x in bl["max_gap"]) == r["max_gap"]
    for i in range(len(bl)):
        a = lo + (i << 20)
        b = min(hi, a + (1 << 20))
        s = orc.sieve_range(a, b)
        for k in ("pi", "twins", "max_gap", "gap_start", "tuple6", "first_prime", "last_prime"):
            assert int(bl[i][k]) == s[k], (i, k)


def test_mutations_are_caught(orc):
    """A planted mistake (one bit of the bitmap flipped) changes the segment hash and the
    count; the comparisons the GPU tests make would catch it."""
    lo, hi = 10 ** 9, 10 ** 9 + 2 ** 20
    r = orc.sieve_range(lo, hi, hash_log2=18, bitmap=True)
    bm = r["bitmap"].copy()
    by = bm.view(np.uint8)
    seg0 = by[: (1 << 17) // 8].copy()
    assert fnv1a64(seg0.tobytes()) == int(r["hashes"][0])
    seg0[100] ^= 0x10
    assert fnv1a64(seg0.tobytes()) != int(r["hashes"][0])
    pop = int(np.unpackbits(by, bitorder="little").sum())
    assert pop == r["pi"]


@pytest.mark.skipif("not __import__('oracle').have_ref()")
def test_oracle_matches_compiled_reference(orc):
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.integers(0, 2 ** 64 - 1, size=100000, dtype=np.uint64),
                         np.arange(0, 5000, dtype=np.uint64)])
    assert np.array_equal(orc.bpsw(xs), orc.ref_bpsw(xs))
    ps = orc.primes_range(10 ** 12, 10 ** 12 + 200000)
    assert np.array_equal(orc.fermat_q(ps), orc.ref_fermat_q(ps))
    big = orc.primes_range(2 ** 62 - 100000, 2 ** 62)
    assert np.array_equal(orc.fermat_q(big), orc.ref_fermat_q(big))
    r = orc.sieve_range(10 ** 15, 10 ** 15 + 2 * 10 ** 9)
    assert (r["tuple6"], r["tuple6_cks"]) == orc.ref_count_sext(10 ** 15, 10 ** 15 + 2 * 10 ** 9)
    w = orc.wieferich_range(10 ** 12, 10 ** 12 + 10 ** 7)
    p, k, f = orc.ref_wieferich_scan(10 ** 12, 10 ** 12 + 10 ** 7)
    assert (w["primes"], w["cks"], f) == (p, k, 0)


@pytest.mark.skipif("not __import__('oracle').have_ref_twins()")
@pytest.mark.parametrize("lo,hi", [(990, 30 * 10 ** 6), (30 * 10 ** 9, 30 * 10 ** 9 + 3 * 10 ** 7),
                                   (999999999999990, 999999999999990 + 6 * 10 ** 7)])
def test_twins_match_reference_twin_sieve(orc, lo, hi):
    """The oracle's twin counts equal those of the reference's own twin-class bucket sieve
    (A007508/a007508.c count_twins_twin), built from the reference's source."""
    assert orc.sieve_range(lo, hi)["twins"] == orc.ref_twins(lo, hi)


def test_config_fixtures_consistent(configs):
    c2 = configs["config2"]
    assert (c2["stats"]["tuple6"], c2["stats"]["tuple6_cks"]) == (c2["reference_tuple6"]["count"],
                                                                   c2["reference_tuple6"]["cks"])
    c4 = configs["config4"]
    assert (c4["primes"], c4["cks"]) == (c4["reference"]["primes"], c4["reference"]["cks"])
    assert c4["flt"] == 0 and c4["tests"] == c4["primes"]
    assert len(configs["config1"]["hashes"]) == 191


def test_mix64_matches_reference_definition(orc):
    for z in [0, 1, 2 ** 63, 2 ** 64 - 1, 12345678901234567]:
        assert orc.mix64(z) == mix64(z)


def test_sieve_near_2_64_against_bpsw(orc):
    """Near the top of the range every sieving prime is close to 2^32: the sieve must agree
    with BPSW run on every odd number."""
    lo = 2 ** 64 - 2 ** 26
    odd = np.arange(lo + 1, lo + 1 + 2 * 300000, 2, dtype=np.uint64)
    r = orc.sieve_range(lo, lo + 600001, bitmap=True)
    v = orc.bpsw(odd)
    bits = np.unpackbits(r["bitmap"].view(np.uint8), bitorder="little")[: len(odd)].astype(bool)
    assert np.array_equal(bits, v) and r["pi"] == int(v.sum())
