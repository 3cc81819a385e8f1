"""Fermat quotients q_p(2) on the GPU through the C ABI against the oracle, the reference's
compiled code, its Python verifier windows and the full-size fixture."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_quotients_vs_oracle(engine, orc):
    for lo, hi in [(3, 100000), (10 ** 12, 10 ** 12 + 10 ** 6), (2 ** 46 - 10 ** 6, 2 ** 46),
                   (2 ** 47 - 10 ** 5, 2 ** 47 + 10 ** 5), (2 ** 62 - 10 ** 5, 2 ** 62), (2 ** 63 - 10 ** 5, 2 ** 63)]:
        p = orc.primes_range(lo, hi)
        p = p[p >= 3]
        assert np.array_equal(engine.fermat_quotient(p), orc.fermat_q(p)), (lo, hi)


def test_known_wieferich_primes(engine, ref_vectors):
    q = engine.fermat_quotient(np.array(ref_vectors["wieferich_base2"], dtype=np.uint64))
    assert (q == 0).all()
    r = engine.wieferich_range(2, 10 ** 6)
    assert r["hits"] == [1093, 3511] and r["flt"] == 0


def test_wieferich_windows_verify_py(engine, verify_py):
    for w in verify_py["wieferich_base2"]:
        r = engine.wieferich_range(w["lo"], w["hi"])
        assert (r["primes"], r["cks"]) == (w["primes"], w["cks"]), w


def test_wieferich_vs_oracle(engine, orc):
    for lo, hi in [(10 ** 12, 10 ** 12 + 10 ** 7), (2 ** 50, 2 ** 50 + 10 ** 6), (3, 10 ** 6)]:
        assert engine.wieferich_range(lo, hi) == orc.wieferich_range(lo, hi), (lo, hi)


def test_config4_fixture(engine, configs):
    c = configs["config4"]
    r = engine.wieferich_range(c["lo"], c["hi"])
    for k in ("primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"):
        assert r[k] == c[k], k
