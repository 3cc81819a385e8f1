"""oracle -- CPU checkers for the Mathpub hot path.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py import this
package, and only to compute expected answers or CPU timings; the product (mathpub_b200)
never does.

  liboracle.so               the C restatement in mp_oracle.c (built by `make` here)
  _ref/libref_a350826.so     the reference's own A350826/a350826.c (BPSW, sextuplet counter)
  _ref/libref_wieferich.so   the reference's own A001220/wieferich.c (Fermat quotients)
The _ref libraries are compiled from the reference tree by `make ref` where that tree
exists, and travel with the repository as built files.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_A350826 = os.path.join(HERE, "_ref", "libref_a350826.so")
REF_A007508 = os.path.join(HERE, "_ref", "libref_a007508.so")
REF_WIEFERICH = os.path.join(HERE, "_ref", "libref_wieferich.so")
# the reference tree (read only to build the checkers): $MATHPUB_REFERENCE, else its checkout on
# the build machine
REFERENCE_TREE = os.environ.get("MATHPUB_REFERENCE", "/root/reference")

STATS_FIELDS = ["pi", "twins", "max_gap", "gap_start", "tuple6", "tuple6_cks", "first_prime", "last_prime"]
STATS_DTYPE = np.dtype([(n, np.uint64) for n in STATS_FIELDS])
TAIL = 1 << 16


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in STATS_FIELDS]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n in STATS_FIELDS}


class Wief(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ["primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"]] + [
        ("hits", C.c_uint64 * 16)]


def build(ref=True):
    """Compile liboracle.so, and the reference checkers when the reference tree exists."""
    target = "ref" if ref and os.path.isdir(REFERENCE_TREE) else "all"
    subprocess.run(["make", "-s", "-C", HERE, target, f"MATHPUB_REFERENCE={REFERENCE_TREE}"], check=True)


_o = None
_ra = None
_rw = None


def o():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        u64, vp = C.c_uint64, C.c_void_p
        for name, args, res in [
            ("or_mix64", [u64], u64),
            ("or_bpsw", [u64], C.c_int), ("or_sprp2", [u64], C.c_int), ("or_slprp", [u64], C.c_int),
            ("or_is_prime_ref", [u64], C.c_int),
            ("or_bpsw_batch", [vp, C.c_size_t, vp, C.c_int], None),
            ("or_fermat_q2", [u64, vp, vp], u64),
            ("or_fermat_batch", [vp, C.c_size_t, vp, C.c_int], None),
            ("or_sieve_range", [u64, u64, u64, C.c_int, C.c_int, vp, vp, vp, vp, C.c_int], C.c_int),
            ("or_primes_range", [u64, u64, vp, C.c_size_t, C.c_int], C.c_size_t),
            ("or_wieferich_range", [u64, u64, vp, C.c_int], C.c_int),
            ("or_fnv1a64", [vp, C.c_size_t], u64),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _o = L
    return _o


def have_ref():
    return os.path.exists(REF_A350826) and os.path.exists(REF_WIEFERICH)


def ra():
    global _ra
    if _ra is None:
        L = C.CDLL(REF_A350826)
        u64, vp = C.c_uint64, C.c_void_p
        for name, args, res in [("ref_bpsw", [u64], C.c_int), ("ref_sprp2_64", [u64], C.c_int),
                                ("ref_slprp64", [u64], C.c_int), ("ref_is_prime", [u64], C.c_int),
                                ("ref_bpsw_batch", [vp, C.c_size_t, vp, C.c_int], None),
                                ("ref_count_sext", [u64, u64, C.c_int, vp, vp], C.c_int)]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _ra = L
    return _ra


_rt = None


def have_ref_twins():
    return os.path.exists(REF_A007508)


def rt():
    """the reference's own twin-class sieve (A007508/a007508.c count_twins_twin)"""
    global _rt
    if _rt is None:
        L = C.CDLL(REF_A007508)
        L.ref_twins_k.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
        L.ref_twins_k.restype = C.c_uint64
        _rt = L
    return _rt


def ref_twins(lo, hi, nthreads=None):
    """Twin pairs (p, p + 2) with lo <= p < hi by the reference's twin sieve; lo, hi multiples
    of 30 and lo > 5 (its k-space: p = 30 k + 11, 17 or 29)."""
    assert lo % 30 == 0 and hi % 30 == 0 and lo > 5
    return int(rt().ref_twins_k(lo // 30, hi // 30, nthreads or threads()))


def rw():
    global _rw
    if _rw is None:
        L = C.CDLL(REF_WIEFERICH)
        u64, vp = C.c_uint64, C.c_void_p
        for name, args, res in [("ref_fermat_q2", [u64, vp, vp], u64),
                                ("ref_fermat_batch", [vp, C.c_size_t, vp, C.c_int], None),
                                ("ref_wieferich_scan", [u64, u64, C.c_int, vp, vp, vp], C.c_int)]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _rw = L
    return _rw


def threads():
    return max(1, os.cpu_count() or 1)


# ---- convenience wrappers ----

def bpsw(n, nthreads=None):
    n = np.ascontiguousarray(n, dtype=np.uint64)
    bits = np.zeros((len(n) + 7) // 8 + 8, dtype=np.uint8)
    o().or_bpsw_batch(n.ctypes.data, len(n), bits.ctypes.data, nthreads or threads())
    return np.unpackbits(bits, bitorder="little")[: len(n)].astype(bool)


def ref_bpsw(n, nthreads=None):
    n = np.ascontiguousarray(n, dtype=np.uint64)
    bits = np.zeros((len(n) + 7) // 8 + 8, dtype=np.uint8)
    ra().ref_bpsw_batch(n.ctypes.data, len(n), bits.ctypes.data, nthreads or threads())
    return np.unpackbits(bits, bitorder="little")[: len(n)].astype(bool)


def fermat_q(p, nthreads=None):
    p = np.ascontiguousarray(p, dtype=np.uint64)
    q = np.zeros(len(p), dtype=np.uint64)
    o().or_fermat_batch(p.ctypes.data, len(p), q.ctypes.data, nthreads or threads())
    return q


def ref_fermat_q(p, nthreads=None):
    p = np.ascontiguousarray(p, dtype=np.uint64)
    q = np.zeros(len(p), dtype=np.uint64)
    rw().ref_fermat_batch(p.ctypes.data, len(p), q.ctypes.data, nthreads or threads())
    return q


def sieve_range(lo, hi, block_log2=0, hash_log2=0, bitmap=False, nthreads=None):
    st = Stats()
    nb = ((hi - lo - 1) >> block_log2) + 1 if block_log2 else 0
    base = lo & ~1
    nbits = (hi - base) >> 1
    nh = (nbits + (1 << (hash_log2 - 1)) - 1) >> (hash_log2 - 1) if hash_log2 else 0
    blocks = np.zeros(nb, dtype=STATS_DTYPE) if block_log2 else None
    hashes = np.zeros(nh, dtype=np.uint64) if hash_log2 else None
    bm = np.zeros((nbits + 63) // 64, dtype=np.uint64) if bitmap else None
    rc = o().or_sieve_range(lo, hi, TAIL, block_log2, hash_log2, C.byref(st),
                            None if blocks is None else blocks.ctypes.data,
                            None if hashes is None else hashes.ctypes.data,
                            None if bm is None else bm.ctypes.data, nthreads or threads())
    if rc != 0:
        raise RuntimeError(f"or_sieve_range failed: {rc}")
    r = st.as_dict()
    if blocks is not None:
        r["blocks"] = blocks
    if hashes is not None:
        r["hashes"] = hashes
    if bm is not None:
        r["bitmap"] = bm
    return r


def primes_range(lo, hi, nthreads=None):
    cap = max(16, (hi - lo) // 2 + 16)
    out = np.zeros(cap, dtype=np.uint64)
    n = o().or_primes_range(lo, hi, out.ctypes.data, cap, nthreads or threads())
    return out[:n]


def wieferich_range(lo, hi, nthreads=None):
    w = Wief()
    rc = o().or_wieferich_range(lo, hi, C.byref(w), nthreads or threads())
    if rc != 0:
        raise RuntimeError("or_wieferich_range failed")
    d = {n: int(getattr(w, n)) for n in ["primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"]}
    d["hits"] = [int(w.hits[i]) for i in range(min(16, d["nhits"]))]
    return d


def ref_count_sext(lo, hi, nthreads=None):
    c, k = C.c_uint64(), C.c_uint64()
    ra().ref_count_sext(lo, hi, nthreads or threads(), C.byref(c), C.byref(k))
    return int(c.value), int(k.value)


def ref_wieferich_scan(lo, hi, nthreads=None):
    p, k, f = C.c_uint64(), C.c_uint64(), C.c_uint64()
    rw().ref_wieferich_scan(lo, hi, nthreads or threads(), C.byref(p), C.byref(k), C.byref(f))
    return int(p.value), int(k.value), int(f.value)


def mix64(z):
    return int(o().or_mix64(z))


GAP_BINS, RUN_MAX, CHAIN_MAX, GAP_LOOK = 1024, 64, 32, 1 << 16


def gap_stats(lo, hi, nthreads=None):
    """Statistics of the gaps that follow the primes p in [lo, hi) (the primes after hi come
    from a look-ahead of 2^16 integers):
      gap_hist[g // 2]  primes whose next gap is g (the gap 1 of p = 2 in bin 0);
      run_hist[L]       primes with L(p) = L, the number of strictly increasing gaps that
                        follow p (A158939/a158939.c:17-30: L(p) = largest n with
                        g_1 < g_2 < ... < g_n);
      run_first[L]      the smallest such p (0 if none): A158939's a(L) on [lo, hi);
      unsettled         primes whose run is still increasing at the end of the look-ahead.
    Computed from the oracle's prime list."""
    p = primes_range(lo, hi + GAP_LOOK, nthreads).astype(np.int64)
    n_in = int(np.searchsorted(p, hi))
    g = np.diff(p)                                    # g[i] = gap after p[i]
    hist = np.zeros(GAP_BINS, dtype=np.uint64)
    gi = g[:n_in] // 2
    hist += np.bincount(np.minimum(gi, GAP_BINS - 1), minlength=GAP_BINS).astype(np.uint64)
    unsettled = n_in - min(n_in, len(g))              # an in-range prime with no next prime
    # run of p[i]: L = 1 + number of consecutive increases g[i] < g[i+1] < ... ; the run of
    # p[i] ends at the first j >= i with g[j + 1] <= g[j]
    stop = np.flatnonzero(g[1:] <= g[:-1])            # j with g[j + 1] <= g[j]
    idx = np.arange(min(n_in, len(g)))
    k = np.searchsorted(stop, idx)                    # first stop >= i
    ended = k < len(stop)
    L = np.where(ended, stop[np.minimum(k, len(stop) - 1)] - idx + 1 if len(stop) else 0, 0)
    unsettled += int((~ended).sum())
    L = L[ended]
    P = p[:len(idx)][ended]
    run_hist = np.zeros(RUN_MAX, dtype=np.uint64)
    run_first = np.zeros(RUN_MAX, dtype=np.uint64)
    Lc = np.minimum(L, RUN_MAX - 1)
    run_hist += np.bincount(Lc, minlength=RUN_MAX).astype(np.uint64)
    for l in range(1, RUN_MAX):                       # P is increasing: the first index is the smallest p
        if run_hist[l]:
            run_first[l] = P[int(np.argmax(Lc == l))]
    cl = chain_lengths(g, len(idx))
    chain_hist = np.bincount(np.minimum(cl, CHAIN_MAX - 1), minlength=CHAIN_MAX).astype(np.uint64)
    return {"gap_hist": hist, "run_hist": run_hist, "run_first": run_first, "unsettled": int(unsettled),
            "chain_hist": chain_hist}


def chain_lengths(g, n):
    """For the first n primes of a list with gaps g: the number of primes in the chain that each
    heads, the m-th gap being 2m (gapchain/gapchain_ps.c:336-342: len = 1 + the gaps 2, 4, 6, ...
    that follow p), up to CHAIN_MAX - 1 gaps."""
    cl = np.ones(n, dtype=np.int64)
    alive = np.ones(n, dtype=bool)
    for m in range(1, CHAIN_MAX):
        j = np.arange(n) + (m - 1)
        ok = j < len(g)
        step = np.zeros(n, dtype=bool)
        step[ok] = g[j[ok]] == 2 * m
        alive &= step
        if not alive.any():
            break
        cl += alive
    return cl


def gap_chains(lo, hi, min_len, nthreads=None):
    """Heads p in [lo, hi) of chains of at least min_len primes with gaps 2, 4, 6, ..., and the
    chain lengths (capped at CHAIN_MAX - 1), in increasing order."""
    p = primes_range(lo, hi + GAP_LOOK, nthreads).astype(np.int64)
    n_in = int(np.searchsorted(p, hi))
    cl = chain_lengths(np.diff(p), n_in)
    sel = cl >= min_len
    return p[:n_in][sel].astype(np.uint64), np.minimum(cl[sel], CHAIN_MAX - 1).astype(np.uint32)


def dec_chains(lo, hi, k, nthreads=None):
    """Chains of at least k consecutive primes with gaps ..., 6, 4, 2 (A263049), as
    gapchain/gapchain_ps.c:365-395 finds them: each exact k-prime pattern p, p + 2(k-1), ...,
    p + (k-1)k of consecutive primes (gaps 2(k-1), ..., 4, 2) with p in [lo, hi) ends a chain,
    which is extended backwards while the gap before its first prime is 2 len.
    Returns (first primes ascending, lengths capped at CHAIN_MAX - 1, keys p)."""
    back = 2 * CHAIN_MAX * CHAIN_MAX
    p = primes_range(max(0, lo - back), hi + GAP_LOOK, nthreads).astype(np.int64)
    g = np.diff(p)
    i0, n_in = int(np.searchsorted(p, lo)), int(np.searchsorted(p, hi))
    idx = np.arange(i0, n_in)
    ok = np.ones(len(idx), dtype=bool)
    for j in range(k - 1):
        t = idx + j
        good = t < len(g)
        step = np.zeros(len(idx), dtype=bool)
        step[good] = g[t[good]] == 2 * (k - 1 - j)
        ok &= step
    heads, lens, keys = [], [], []
    for i in idx[ok]:
        h, n = int(i), k
        while n < CHAIN_MAX - 1 and h > 0 and g[h - 1] == 2 * n:
            h -= 1
            n += 1
        heads.append(int(p[h]))
        lens.append(n)
        keys.append(int(p[i]))
    o = np.argsort(np.array(heads, dtype=np.uint64), kind="stable")
    return (np.array(heads, dtype=np.uint64)[o], np.array(lens, dtype=np.uint32)[o],
            np.array(keys, dtype=np.uint64)[o])
