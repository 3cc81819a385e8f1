"""mathpub_b200 -- Python binding of libmathpub, the B200 (sm_100a) engine for the Mathpub
integer hot path (segmented sieve and scans, 64-bit BPSW, Fermat quotients mod p^2).

The compute lives in hand-written CUDA kernels behind the C ABI of include/mathpub_gpu.h;
this module only loads the in-tree libmathpub.so with ctypes, moves numpy arrays across the
boundary and turns status codes into exceptions.  There is no CPU fallback: if the library
or a GPU is missing, every call raises.

Names follow the reference tools (paths inside the Mathpub project):
    Engine.bpsw                 bpsw()             A350826/a350826.c:965
    Engine.sieve_range          the segment sieve and its scans (count, twins, gaps, 6-tuples)
    Engine.fermat_quotient      fermat_quotient()  A001220/wieferich.c:939 (base 2)
    Engine.wieferich_range      scan_chunk()       A001220/wieferich.c:1129 (base 2)
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmathpub.so")
WORK_PATH = os.path.join(HERE, "libmpwork.so")

MP_OK, MP_EINVAL, MP_ENOMEM, MP_ECUDA, MP_ETIMEOUT, MP_EOVERFLOW, MP_ERANGE, MP_EAGAIN, MP_EBUSY = 0, -1, -2, -3, -4, -5, -6, -7, -8
MODE_BATCHED, MODE_PLAIN = 0, 1
_ERRNAMES = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ETIMEOUT", -5: "EOVERFLOW", -6: "ERANGE", -7: "EAGAIN", -8: "EBUSY"}

# largest count mp_wieferich_stats_noalloc accepts (MP_NOALLOC_MAX_COUNT in include/mathpub_gpu.h)
NOALLOC_MAX_COUNT = 1 << 24

STATS_FIELDS = ["pi", "twins", "max_gap", "gap_start", "tuple6", "tuple6_cks", "first_prime", "last_prime"]
WIEF_FIELDS = ["primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"]


class RangeStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in STATS_FIELDS]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n in STATS_FIELDS}


class SieveOpts(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("tile_log2", C.c_uint32), ("block_log2", C.c_uint32),
                ("hash_log2", C.c_uint32), ("threads", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class WiefStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in WIEF_FIELDS] + [("hits", C.c_uint64 * 16)]

    def as_dict(self):
        d = {n: int(getattr(self, n)) for n in WIEF_FIELDS}
        d["hits"] = [int(self.hits[i]) for i in range(min(16, d["nhits"]))]
        return d


STATS_DTYPE = np.dtype([(n, np.uint64) for n in STATS_FIELDS])


class ServeOpts(C.Structure):
    _fields_ = [("mem_budget", C.c_uint64), ("max_inflight", C.c_uint32), ("streams", C.c_uint32),
                ("prime_limit", C.c_uint64), ("chunk", C.c_uint64)]


class ServeResult(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("status", C.c_int32), ("pi", C.c_uint64), ("max_gap", C.c_uint64),
                ("gap_start", C.c_uint64), ("twins", C.c_uint64), ("count", C.c_uint32),
                ("submit_s", C.c_double), ("done_s", C.c_double)]


GAP_BINS, RUN_MAX, CHAIN_MAX = 1024, 64, 32


class GapStats(C.Structure):
    _fields_ = [("gap_hist", C.c_uint64 * GAP_BINS), ("run_hist", C.c_uint64 * RUN_MAX),
                ("run_first", C.c_uint64 * RUN_MAX), ("unsettled", C.c_uint64), ("chain_hist", C.c_uint64 * CHAIN_MAX)]

    def as_dict(self):
        return {"gap_hist": np.ctypeslib.as_array(self.gap_hist).copy(),
                "run_hist": np.ctypeslib.as_array(self.run_hist).copy(),
                "run_first": np.ctypeslib.as_array(self.run_first).copy(), "unsettled": int(self.unsettled),
                "chain_hist": np.ctypeslib.as_array(self.chain_hist).copy()}


class MathpubError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None
_work = None


def lib():
    """The loaded libmathpub.so (built in-tree by mathpub_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MathpubError(MP_EINVAL, f"{LIB_PATH} is missing: run `python -m mathpub_b200.build`")
        L = C.CDLL(LIB_PATH)
        u64, u32, vp = C.c_uint64, C.c_uint32, C.c_void_p
        sig = {
            "mp_init": ([C.c_int, C.POINTER(vp)], C.c_int),
            "mp_free": ([vp], C.c_int),
            "mp_last_error": ([vp], C.c_char_p),
            "mp_version": ([], C.c_int),
            "mp_last_kernel_ms": ([vp], C.c_double),
            "mp_sieve_nblocks": ([u64, u64, u32], u64),
            "mp_sieve_nhashes": ([u64, u64, u32], u64),
            "mp_sieve_nwords": ([u64, u64], u64),
            "mp_sieve_range": ([vp, u64, u64, vp, vp, vp, vp, vp], C.c_int),
            "mp_sieve_range_dev": ([vp, u64, u64, vp, vp, vp, vp, vp, vp], C.c_int),
            "mp_primes_range": ([vp, u64, u64, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
            "mp_bpsw_u64": ([vp, vp, C.c_size_t, vp], C.c_int),
            "mp_bpsw_batches": ([vp, vp, vp, u32, vp], C.c_int),
            "mp_bpsw_lists_dev": ([vp, vp, vp, vp, u32, vp, u32, vp], C.c_int),
            "mp_fermat_q_base2": ([vp, vp, C.c_size_t, vp], C.c_int),
            "mp_fermat_q_base2_dev": ([vp, vp, C.c_size_t, vp, vp], C.c_int),
            "mp_wieferich_range": ([vp, u64, u64, vp], C.c_int),
            "mp_wieferich_stats_noalloc": ([vp, vp, u64, vp, vp], C.c_int),
            "mp_gap_stats_range": ([vp, u64, u64, vp], C.c_int),
            "mp_gap_chains": ([vp, u64, u64, u32, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
            "mp_chain_sieve": ([vp, u64, u64, u32, u32, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
            "mp_tuple_count": ([vp, u64, u64, vp, u32, C.POINTER(u64), C.POINTER(u64)], C.c_int),
            "mp_tuple_count128": ([vp, vp, vp, vp, u32, C.POINTER(u64), C.POINTER(u64)], C.c_int),
            "mp_chain_first": ([vp, u64, u64, u32, u32, C.POINTER(u64), C.POINTER(u64), C.POINTER(u32)], C.c_int),
            "mp_chain_sieve128": ([vp, vp, vp, u32, u32, vp, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
            "mp_chain_first128": ([vp, vp, vp, u32, u32, vp, vp, C.POINTER(u32)], C.c_int),
            "mp_autotune": ([vp, u64, C.c_char_p, C.c_size_t], C.c_int),
            "mp_tune_set": ([vp, C.c_int, C.c_int], C.c_int),
            "mp_profile_enable": ([vp, C.c_int], C.c_int),
            "mp_profile_read": ([vp, vp, vp, C.c_int], C.c_int),
            "mp_probe_peaks": ([vp] + [C.POINTER(C.c_double)] * 4, C.c_int),
            "mp_serve_open": ([vp, vp, C.POINTER(vp)], C.c_int),
            "mp_serve_submit_range": ([vp, u64, u64, C.POINTER(u64)], C.c_int),
            "mp_serve_submit_bpsw": ([vp, vp, u32, vp, C.POINTER(u64)], C.c_int),
            "mp_serve_poll": ([vp, u64, vp, C.c_int], C.c_int),
            "mp_serve_close": ([vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def work():
    """libmpwork.so: the seeded workload generators (plain C, no GPU)."""
    global _work
    if _work is None:
        if not os.path.exists(WORK_PATH):
            raise MathpubError(MP_EINVAL, f"{WORK_PATH} is missing: run `python -m mathpub_b200.build`")
        W = C.CDLL(WORK_PATH)
        W.mpw_bpsw_batch.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p]
        W.mpw_bpsw_batch.restype = C.c_int
        W.mpw_uniform_odd.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p]
        W.mpw_uniform_odd.restype = None
        _work = W
    return _work


def bpsw_workload(seed, count, nlists):
    """The seeded BPSW batch: (candidates uint64[count], list lengths uint32[nlists])."""
    n = np.empty(count, dtype=np.uint64)
    lens = np.empty(max(nlists, 1), dtype=np.uint32)
    if work().mpw_bpsw_batch(seed, count, nlists, n.ctypes.data, lens.ctypes.data) != 0:
        raise MathpubError(MP_EINVAL, "workload generation failed")
    return n, lens[:nlists]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Engine:
    """One libmathpub handle on one device."""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        rc = lib().mp_init(device, C.byref(self._h))
        if rc != MP_OK:
            raise MathpubError(rc, f"mp_init({device}) failed (no usable CUDA device?)")

    def close(self):
        if self._h:
            lib().mp_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        if rc != MP_OK:
            raise MathpubError(rc, lib().mp_last_error(self._h).decode(errors="replace"))

    def last_kernel_ms(self):
        return lib().mp_last_kernel_ms(self._h)

    # ---- sieve ----
    def sieve_range(self, lo, hi, block_log2=0, hash_log2=0, bitmap=False, mode=MODE_BATCHED, tile_log2=0,
                    threads=0):
        o = SieveOpts(mode, tile_log2, block_log2, hash_log2, threads)
        out = RangeStats()
        L = lib()
        nb = L.mp_sieve_nblocks(lo, hi, block_log2) if block_log2 else 0
        nh = L.mp_sieve_nhashes(lo, hi, hash_log2) if hash_log2 else 0
        nw = L.mp_sieve_nwords(lo, hi) if bitmap else 0
        blocks = np.zeros(nb, dtype=STATS_DTYPE) if block_log2 else None
        hashes = np.zeros(nh, dtype=np.uint64) if hash_log2 else None
        bm = np.zeros(nw, dtype=np.uint64) if bitmap else None
        self._check(L.mp_sieve_range(self._h, lo, hi, C.byref(o), C.byref(out), _p(blocks if nb else None),
                                     _p(hashes if nh else None), _p(bm if nw else None)))
        r = out.as_dict()
        if blocks is not None:
            r["blocks"] = blocks
        if hashes is not None:
            r["hashes"] = hashes
        if bm is not None:
            r["bitmap"] = bm
        return r

    def primes_range(self, lo, hi):
        L = lib()
        cnt = C.c_size_t(0)
        self._check(L.mp_primes_range(self._h, lo, hi, None, 0, C.byref(cnt)))
        out = np.empty(cnt.value, dtype=np.uint64)
        self._check(L.mp_primes_range(self._h, lo, hi, _p(out), cnt.value, C.byref(cnt)))
        return out

    # ---- BPSW ----
    def bpsw(self, n):
        """Verdicts (bool array) for uint64 candidates n."""
        n = np.ascontiguousarray(n, dtype=np.uint64)
        bits = np.zeros((len(n) + 7) // 8 + 8, dtype=np.uint8)
        self._check(lib().mp_bpsw_u64(self._h, _p(n), len(n), _p(bits)))
        return np.unpackbits(bits, bitorder="little")[: len(n)].astype(bool)

    def bpsw_batches(self, lists):
        lists = [np.ascontiguousarray(x, dtype=np.uint64) for x in lists]
        k = len(lists)
        outs = [np.zeros((len(x) + 7) // 8 + 8, dtype=np.uint8) for x in lists]
        lp = (C.c_void_p * k)(*[x.ctypes.data for x in lists])
        op = (C.c_void_p * k)(*[o.ctypes.data for o in outs])
        lens = np.array([len(x) for x in lists], dtype=np.uint32)
        self._check(lib().mp_bpsw_batches(self._h, lp, _p(lens), k, op))
        return [np.unpackbits(o, bitorder="little")[: len(x)].astype(bool) for o, x in zip(outs, lists)]

    # ---- Fermat ----
    def fermat_quotient(self, p):
        p = np.ascontiguousarray(p, dtype=np.uint64)
        q = np.zeros(len(p), dtype=np.uint64)
        self._check(lib().mp_fermat_q_base2(self._h, _p(p), len(p), _p(q)))
        return q

    def gap_stats(self, lo, hi):
        """Gap histogram and A158939 run statistics of the primes in [lo, hi)
        (mp_gap_stats_range)."""
        g = GapStats()
        self._check(lib().mp_gap_stats_range(self._h, lo, hi, C.byref(g)))
        return g.as_dict()

    def gap_chains(self, lo, hi, min_len):
        """Heads p in [lo, hi) of chains of at least min_len primes with gaps 2, 4, 6, ... and the
        chain lengths (mp_gap_chains), in increasing order."""
        n = C.c_size_t()
        self._check(lib().mp_gap_chains(self._h, lo, hi, min_len, None, None, 0, C.byref(n)))
        heads = np.zeros(max(1, n.value), dtype=np.uint64)
        lens = np.zeros(max(1, n.value), dtype=np.uint32)
        self._check(lib().mp_gap_chains(self._h, lo, hi, min_len, _p(heads), _p(lens), n.value, C.byref(n)))
        return heads[:n.value], lens[:n.value]

    def chain_sieve(self, lo, hi, k, dec=False):
        """Chains of at least k consecutive primes by the constellation sieve (mp_chain_sieve):
        gaps 2, 4, 6, ... (the same heads and lengths as gap_chains), or with dec=True gaps
        ..., 6, 4, 2, keyed by the k-prime pattern that ends the chain and reported from the
        chain's first prime.  Returns (heads, lens) in ascending order of head."""
        n = C.c_size_t()
        shape = 1 if dec else 0
        self._check(lib().mp_chain_sieve(self._h, lo, hi, k, shape, None, None, 0, C.byref(n)))
        heads = np.zeros(max(1, n.value), dtype=np.uint64)
        lens = np.zeros(max(1, n.value), dtype=np.uint32)
        self._check(lib().mp_chain_sieve(self._h, lo, hi, k, shape, _p(heads), _p(lens), n.value, C.byref(n)))
        return heads[:n.value], lens[:n.value]

    def chain_first(self, lo, hi, k, dec=False):
        """The first chain of at least k primes with its key in [lo, hi) (mp_chain_first):
        (key, first prime, length), or None when there is none."""
        key, head, n = C.c_uint64(), C.c_uint64(), C.c_uint32()
        self._check(lib().mp_chain_first(self._h, lo, hi, k, 1 if dec else 0, C.byref(key), C.byref(head),
                                         C.byref(n)))
        return (key.value, head.value, n.value) if n.value else None

    @staticmethod
    def _w2(x):
        return np.array([x & (2 ** 64 - 1), x >> 64], dtype=np.uint64)

    def chain_sieve128(self, lo, hi, k, dec=False):
        """chain_sieve for 128-bit ranges (mp_chain_sieve128, hi <= 3.3e24): a list of
        (first prime, length) with Python integers, ascending."""
        shape = 1 if dec else 0
        wl, wh = self._w2(lo), self._w2(hi)
        n = C.c_size_t()
        self._check(lib().mp_chain_sieve128(self._h, _p(wl), _p(wh), k, shape, None, None, 0, C.byref(n)))
        heads = np.zeros(2 * max(1, n.value), dtype=np.uint64)
        lens = np.zeros(max(1, n.value), dtype=np.uint32)
        self._check(lib().mp_chain_sieve128(self._h, _p(wl), _p(wh), k, shape, _p(heads), _p(lens), n.value,
                                            C.byref(n)))
        return [(int(heads[2 * i]) | int(heads[2 * i + 1]) << 64, int(lens[i])) for i in range(n.value)]

    def chain_first128(self, lo, hi, k, dec=False):
        """chain_first for 128-bit ranges (mp_chain_first128): (key, first prime, length) or None."""
        wl, wh = self._w2(lo), self._w2(hi)
        key, head = np.zeros(2, dtype=np.uint64), np.zeros(2, dtype=np.uint64)
        n = C.c_uint32()
        self._check(lib().mp_chain_first128(self._h, _p(wl), _p(wh), k, 1 if dec else 0, _p(key), _p(head),
                                            C.byref(n)))
        if not n.value:
            return None
        return int(key[0]) | int(key[1]) << 64, int(head[0]) | int(head[1]) << 64, n.value

    def tuple_count(self, lo, hi, offs):
        """(count, checksum) of the p in [lo, hi) with p + o prime for every o in offs
        (mp_tuple_count; offs starts at 0, even and increasing)."""
        o = np.ascontiguousarray(offs, dtype=np.uint32)
        n, c = C.c_uint64(), C.c_uint64()
        self._check(lib().mp_tuple_count(self._h, lo, hi, _p(o), len(o), C.byref(n), C.byref(c)))
        return n.value, c.value

    def tuple_count128(self, lo, hi, offs):
        """tuple_count for 128-bit ranges (mp_tuple_count128, hi <= 3.3e24): (count, checksum)."""
        o = np.ascontiguousarray(offs, dtype=np.uint32)
        wl, wh = self._w2(lo), self._w2(hi)
        n, c = C.c_uint64(), C.c_uint64()
        self._check(lib().mp_tuple_count128(self._h, _p(wl), _p(wh), _p(o), len(o), C.byref(n), C.byref(c)))
        return n.value, c.value

    def wieferich_range(self, lo, hi):
        out = WiefStats()
        self._check(lib().mp_wieferich_range(self._h, lo, hi, C.byref(out)))
        return out.as_dict()

    PROF_CATS = ["scatter", "tile", "fold", "hash", "bpsw_batched", "bpsw_plain", "fermat", "fermat_stats", "pipeline"]

    def profile(self, on=True):
        self._check(lib().mp_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        n = len(self.PROF_CATS)
        la = np.zeros(n, dtype=np.uint64)
        ms = np.zeros(n, dtype=np.float64)
        self._check(lib().mp_profile_read(self._h, _p(la), _p(ms), n))
        return {c: (int(la[i]), float(ms[i])) for i, c in enumerate(self.PROF_CATS)}

    def probe_peaks(self):
        a, b, c, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self._check(lib().mp_probe_peaks(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"smem_atomic_conflict_free": a.value, "smem_atomic_random": b.value, "imad32": c.value,
                "l2_atomic_random": d.value}

    TUNE_KNOBS = {"tile_log2": 1, "threads": 2, "scatter_staged": 3, "bucket_div": 4, "no_pipeline": 5,
                  "bpsw_variant": 6, "fermat_ilp2": 7}

    def tune_set(self, **knobs):
        """Pin autotuner choices on this engine, e.g. tune_set(bucket_div=2, no_pipeline=1)."""
        for k, v in knobs.items():
            self._check(lib().mp_tune_set(self._h, self.TUNE_KNOBS[k], int(v)))

    def autotune(self, lo=10**15):
        buf = C.create_string_buffer(4096)
        self._check(lib().mp_autotune(self._h, lo, buf, 4096))
        return buf.value.decode()


class Server:
    """Continuous-batching request server on an Engine (mp_serve_*)."""

    def __init__(self, engine, streams=4, max_inflight=256, mem_budget=0, prime_limit=0, chunk=0):
        self.e = engine
        self._s = C.c_void_p()
        o = ServeOpts(mem_budget, max_inflight, streams, prime_limit, chunk)
        engine._check(lib().mp_serve_open(engine.handle, C.byref(o), C.byref(self._s)))
        self._bits = {}

    def submit_range(self, lo, hi):
        rid = C.c_uint64()
        rc = lib().mp_serve_submit_range(self._s, lo, hi, C.byref(rid))
        if rc != MP_OK:
            raise MathpubError(rc, f"submit_range({lo}, {hi})")
        return rid.value

    def submit_bpsw(self, n):
        n = np.ascontiguousarray(n, dtype=np.uint64)
        bits = np.zeros((len(n) + 7) // 8 + 8, dtype=np.uint8)
        rid = C.c_uint64()
        rc = lib().mp_serve_submit_bpsw(self._s, _p(n), len(n), _p(bits), C.byref(rid))
        if rc != MP_OK:
            raise MathpubError(rc, "submit_bpsw")
        self._bits[rid.value] = (bits, len(n))
        return rid.value

    def poll(self, rid, wait_ms=0):
        """None while pending; else a dict (range: pi, max_gap, gap_start, twins; primality:
        'verdicts' bool array) with 'submit_s', 'done_s' and 'status'."""
        r = ServeResult()
        rc = lib().mp_serve_poll(self._s, rid, C.byref(r), wait_ms)
        if rc == MP_EAGAIN:
            return None
        if rc != MP_OK:
            raise MathpubError(rc, f"poll({rid})")
        d = {"kind": r.kind, "status": r.status, "submit_s": r.submit_s, "done_s": r.done_s}
        if r.kind == 1:
            d.update(pi=int(r.pi), max_gap=int(r.max_gap), gap_start=int(r.gap_start), twins=int(r.twins))
        else:
            bits, n = self._bits.pop(rid)
            d["verdicts"] = np.unpackbits(bits, bitorder="little")[:n].astype(bool)
        return d

    def close(self):
        if self._s:
            lib().mp_serve_close(self._s)
            self._s = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
