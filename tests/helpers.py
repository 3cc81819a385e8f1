"""Small pure-Python definitions used by the tests (trial-division truth for tiny ranges,
FNV-1a-64)."""
import numpy as np

FNV_OFF, FNV_PRIME, M64 = 0xcbf29ce484222325, 0x100000001b3, (1 << 64) - 1


def is_prime_td(n):
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    d = 3
    while d * d <= n:
        if n % d == 0:
            return False
        d += 2
    return True


def fnv1a64(data):
    h = FNV_OFF
    for c in bytes(data):
        h = ((h ^ c) * FNV_PRIME) & M64
    return h


def brute_range(lo, hi, block_log2=0, hash_log2=0):
    """The range definitions of include/mathpub_gpu.h evaluated by trial division (tiny ranges)."""
    def nextprime(p):
        q = p + 1
        while not is_prime_td(q):
            q += 1
        return q

    primes = [p for p in range(lo, hi) if is_prime_td(p)]
    r = {"pi": len(primes), "twins": sum(is_prime_td(p + 2) for p in primes)}
    tup = [p for p in primes if all(is_prime_td(p + d) for d in (4, 6, 10, 12, 16))]
    r["tuple6"] = len(tup)
    r["first_prime"] = primes[0] if primes else 0
    r["last_prime"] = primes[-1] if primes else 0
    mg, ms = 0, 0
    for p in primes:
        g = nextprime(p) - p
        if g > mg:
            mg, ms = g, p
    r["max_gap"], r["gap_start"] = mg, ms
    base = lo & ~1
    nbits = (hi - base) >> 1
    bits = np.zeros(nbits, dtype=np.uint8)
    for i in range(nbits):
        bits[i] = is_prime_td(base + 2 * i + 1)
    r["bits"] = bits
    if hash_log2:
        sb = 1 << (hash_log2 - 1)
        hs = []
        for s in range(0, nbits, sb):
            seg = bits[s:s + sb]
            hs.append(fnv1a64(np.packbits(seg, bitorder="little").tobytes()))
        r["hashes"] = hs
    return r


GOLD = 0x9E3779B97F4A7C15


def mix64(z):
    z = (z + GOLD) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def tuple6_cks(lo, hi):
    s = 0
    for p in range(lo, hi):
        if is_prime_td(p) and all(is_prime_td(p + d) for d in (4, 6, 10, 12, 16)):
            s = (s + mix64(p)) & M64
    return s
