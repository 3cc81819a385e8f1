"""Prime constellations by the constellation sieve (mp_tuple_count): the number of p with every
p + o prime and the sum of mix64(p), from a search that sieves only the admissible residue
classes, as the reference's A350826 class sieve does (A350826/a350826.c:1522).

GPU: the sextuplets {0, 4, 6, 10, 12, 16} give the reference's A350826(1..13) and its checksum
windows, and equal the full sieve's tuple6 and tuple6_cks; prime quadruplets {0, 2, 6, 8} equal
a count over the oracle's primes; an inadmissible pattern has only its small exception."""
import re

import numpy as np
import pytest

from helpers import mix64

SEXT = [0, 4, 6, 10, 12, 16]
pytestmark = pytest.mark.gpu


def num(s):
    """'1e17-1e12', '2^64+1e12', ... as an integer."""
    return eval(re.sub(r"(\d+)e(\d+)", r"(\1*10**\2)", s).replace("^", "**"), {})


def test_sextuplets_give_a350826(engine, ref_vectors):
    a = ref_vectors["A350826"]
    for n in range(1, 14):
        assert engine.tuple_count(10 ** (n - 1), 10 ** n, SEXT)[0] == a[n], n


def test_sextuplet_windows(engine, ref_vectors):
    """All seven of the reference's checksum windows (A350826/a350826.c:2571), three of them above
    2^64 (2^64 +- 1e12, 1e20 +- 1e12, [1e22, 1e22 + 2e12)), where the checksum term is hashp(p)."""
    checked = 0
    for w in ref_vectors["sext_windows"]:
        lo, hi = num(w["lo"]), num(w["hi"])
        if hi <= 2 ** 64 - 2 ** 12:
            assert engine.tuple_count(lo, hi, SEXT) == (w["count"], w["cks"]), w
        assert engine.tuple_count128(lo, hi, SEXT) == (w["count"], w["cks"]), w
        checked += 1
    assert checked == 7


@pytest.mark.parametrize("lo,hi", [(0, 10 ** 9), (10 ** 12 + 1, 10 ** 12 + 10 ** 11), (2 ** 62 - 10 ** 11, 2 ** 62)])
def test_sextuplets_equal_the_full_sieve(engine, lo, hi):
    r = engine.sieve_range(lo, hi)
    assert engine.tuple_count(lo, hi, SEXT) == (r["tuple6"], r["tuple6_cks"])


def test_quadruplets_equal_the_oracle(engine, orc):
    lo, hi = 0, 10 ** 8
    p = orc.primes_range(lo, hi + 16).astype(np.int64)
    s = set(p.tolist())
    heads = [int(x) for x in p if x < hi and all(int(x) + d in s for d in (2, 6, 8))]
    cks = 0
    for x in heads:
        cks = (cks + mix64(x)) & (2 ** 64 - 1)
    assert engine.tuple_count(lo, hi, [0, 2, 6, 8]) == (len(heads), cks)


def test_inadmissible_pattern_and_errors(engine):
    import mathpub_b200 as mp
    assert engine.tuple_count(0, 10 ** 9, [0, 2, 4]) == (1, mix64(3))     # 3, 5, 7 only
    with pytest.raises(mp.MathpubError):
        engine.tuple_count(0, 100, [2, 4])
    with pytest.raises(mp.MathpubError):
        engine.tuple_count(0, 100, [0, 3])
