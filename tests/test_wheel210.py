"""The wheel of 210 of the staged bucket scatter (mathpub_b200/csrc/mp_sieve.cu): its constant
tables equal their definitions, and the walk they drive (per prime, the first multiple with k
coprime to 210, then six groups of eight progressions of stride 105 q) yields exactly the bits
j < span of the multiples x0 + 2 j = q k >= max(x0, q^2) with gcd(k, 210) = 1.  CPU only."""
import math
import os
import random
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "mathpub_b200", "csrc", "mp_sieve.cu")

RES = [k for k in range(1, 210) if math.gcd(k, 210) == 1]        # the 48 residues, all odd


def table(name):
    text = open(SRC).read()
    m = re.search(r"__constant__ u8 " + name + r"\[(\d+)\] = \{([^}]*)\};", text)
    assert m, name
    vals = [int(x) for x in m.group(2).replace("\n", " ").split(",") if x.strip()]
    assert len(vals) == int(m.group(1))
    return vals


def test_tables_match_their_definitions():
    off, nidx, ndist, inv = (table(n) for n in ("c_w210_off", "c_w210_nidx", "c_w210_ndist", "c_w210_inv"))
    assert len(RES) == 48
    assert off == [(RES[t % 48] + 210 * (t // 48) - 1) // 2 for t in range(96)]
    for km in range(1, 210, 2):                                     # odd k mod 210
        d = next(d for d in range(0, 210, 2) if math.gcd((km + d) % 210, 210) == 1)
        assert RES[nidx[km]] == (km + d) % 210 and ndist[km] == d // 2, km
    for q in range(210):
        if math.gcd(q, 210) == 1:
            assert q * inv[q] % 210 == 1, q


def first_odd_multiple(x0, q, cap):
    """bit j of the first odd multiple x0 + 2 j of q with x0 + 2 j >= max(x0, q^2), capped"""
    r = x0 % q
    d = (q - r) % q
    j = (d + q) // 2 if d % 2 else d // 2
    if q * q > x0:
        j = (q * q - x0) // 2
    return min(j, cap)


def walk(x0, q, span, off, nidx, ndist, inv):
    """the kernel's walk (w210_prime, w210_group and the rounds), on plain integers"""
    j = first_odd_multiple(x0, q, span)
    if j >= span:
        return []
    km = ((x0 % 210) + 2 * (j % 105)) % 210 * inv[q % 210] % 210
    w, jf = nidx[km], j + q * ndist[km]
    if jf >= span:
        return []
    hits = []
    for g in range(6):
        jj = [jf + q * (off[w + 8 * g + i] - off[w]) for i in range(8)]
        if jj[0] >= span:
            break                                                   # later groups start further on
        while jj[0] < span:
            for i in range(8):
                if jj[i] < span:
                    hits.append(jj[i])
                    jj[i] += 105 * q
    return sorted(hits)


def brute(x0, q, span):
    return [j for j in range(span) if (x0 + 2 * j) % q == 0 and x0 + 2 * j >= q * q
            and math.gcd((x0 + 2 * j) // q, 210) == 1]


def test_walk_matches_brute_force():
    tabs = [table(n) for n in ("c_w210_off", "c_w210_nidx", "c_w210_ndist", "c_w210_inv")]
    rng = random.Random(210)
    primes = [p for p in range(11, 3000) if all(p % d for d in range(2, int(p ** 0.5) + 1))]
    for _ in range(1500):
        q = rng.choice(primes)
        x0 = rng.randrange(1, 4 * 10 ** 6) | 1
        span = rng.randrange(1, 30000)
        assert walk(x0, q, span, *tabs) == brute(x0, q, span), (x0, q, span)
