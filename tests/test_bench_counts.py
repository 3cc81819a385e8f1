"""The exact work counts behind bench.py's rooflines, against brute force on small cases (CPU):
the sieve's marks (wheel of 30 below the bucket threshold; bucket records on the staged
scatter's wheel of 210, or the binned scatter's wheel of 30), and the BPSW products (the base-2
ladder's steps, and the Lucas ladder's with two products a step where Selfridge's D is 5)."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def small_primes(n):
    return [p for p in range(3, n) if all(p % d for d in range(2, int(p ** 0.5) + 1))]


def brute_marks(primes, lo, hi, tile_bits, wheel_big):
    top = hi + (1 << 16)
    small = big = 0
    for q in primes:
        if q < 97:
            continue
        wheel = 30 if q <= tile_bits else wheel_big
        k0 = -(-max(lo, q * q) // q)
        k1 = max(-(-top // q), k0)
        n = sum(1 for k in range(k0, k1) if math.gcd(k, wheel) == 1)
        if q <= tile_bits:
            small += n
        else:
            big += n
    return small, big


def test_sieve_marks_on_both_wheels():
    pr = small_primes(3000)
    arr = np.array(pr, dtype=np.uint64)
    lo, hi, tile = 10 ** 6, 10 ** 6 + 200000, 1 << 9
    for staged, wheel in ((True, 210), (False, 30)):
        got = bench.algorithmic_work(arr, lo, hi, tile, staged)
        assert got == tuple(float(x) for x in brute_marks(pr, lo, hi, tile, wheel)), staged


def jacobi(a, n):
    a %= n
    t = 1
    while a:
        while a % 2 == 0:
            a //= 2
            if n % 8 in (3, 5):
                t = -t
        a, n = n, a
        if a % 4 == 3 and n % 4 == 3:
            t = -t
        a %= n
    return t if n == 1 else 0


def selfridge_d(n):
    d = 5
    while True:
        if jacobi(d, n) == -1:
            return d
        d = -(d + 2) if d > 0 else -(d - 2)


def test_bpsw_products_follow_selfridge():
    rng = np.random.default_rng(5)
    n = rng.integers(1 << 20, 1 << 40, size=400, dtype=np.uint64) | np.uint64(1)
    pm = np.array([all(int(x) % d for d in range(3, int(math.isqrt(int(x))) + 1, 2)) for x in n])
    sprp, lucas, surv, nprimes = bench.bpsw_products(n, pm)
    want_sprp = want_lucas = want_surv = 0
    for x, p in zip((int(v) for v in n), pm):
        if x < 131 * 131 or any(x % q == 0 for q in bench.TD_PRIMES):
            continue
        want_surv += 1
        d = x - 1
        while d % 2 == 0:
            d //= 2
        want_sprp += d.bit_length() - 1
        if p:
            e = x + 1
            while e % 2 == 0:
                e //= 2
            per = 2 if selfridge_d(x) == 5 else 4
            assert (per == 2) == (x % 5 in (2, 3))
            want_lucas += per * (e.bit_length() - 1)
    assert (sprp, lucas, surv, nprimes) == (want_sprp, want_lucas, want_surv, int(pm.sum()))
