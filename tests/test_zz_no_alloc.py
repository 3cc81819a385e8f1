"""The allocation-free entry point mp_wieferich_stats_noalloc, called through the C ABI.

Some callers cannot allocate device memory (their framework's allocator owns the device,
or they run where a cudaMalloc, which can synchronise the device, is not allowed).  This
entry point serves them from a fixed scratch array inside the library.  Its results must
equal those of mp_wieferich_range and of the oracle on the same primes, call after call,
because the scratch that one call leaves behind must not leak into the next.

This file is named to be collected last, so that a run stopping at the first failure has
run every other test before it."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"]


def _noalloc(p_dev, q_dev, count, stats_dev, stream):
    import mathpub_b200 as mp
    return mp.lib().mp_wieferich_stats_noalloc(C.c_void_p(p_dev), C.c_void_p(q_dev), count, C.c_void_p(stats_dev),
                                               C.c_void_p(stream))


def _read(stats):
    v = stats.cpu().numpy().view(np.uint64)
    d = dict(zip(FIELDS, [int(x) for x in v[:7]]))
    d["hits"] = [int(x) for x in v[7:7 + min(16, d["nhits"])]]
    d["hit_slots"] = [int(x) for x in v[7:23]]
    return d


def _run_twice(p, q):
    """Two calls in a row on the same arrays; both results."""
    import torch
    import mathpub_b200 as mp
    dev = torch.device("cuda", 0)
    d_p = torch.from_numpy(np.ascontiguousarray(p, dtype=np.uint64).view(np.int64)).to(dev)
    d_q = torch.from_numpy(np.ascontiguousarray(q, dtype=np.uint64).view(np.int64)).to(dev)
    s = torch.cuda.Stream(device=dev)
    out = []
    for _ in range(2):
        stats = torch.full((7 + 16,), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(d_p.data_ptr() if len(p) else 0, d_q.data_ptr() if len(p) else 0, len(p), stats.data_ptr(),
                      s.cuda_stream)
        assert rc == mp.MP_OK
        s.synchronize()
        out.append(_read(stats))
    return out


@pytest.mark.parametrize("lo,hi", [(1000, 4000), (10 ** 12, 10 ** 12 + 10 ** 7)])
def test_noalloc_matches_range_entry_and_oracle(engine, lo, hi):
    import oracle
    want = engine.wieferich_range(lo, hi)
    ref = oracle.wieferich_range(lo, hi)
    for k in FIELDS:
        assert want[k] == ref[k], (k, want[k], ref[k])
    assert want["hits"] == ref["hits"]
    p = engine.primes_range(lo, hi)
    q = engine.fermat_quotient(p)
    for got in _run_twice(p, q):
        for k in FIELDS:
            assert got[k] == ref[k], (k, got[k], ref[k])
        assert got["hits"] == ref["hits"]


def test_noalloc_empty_input(engine):
    for got in _run_twice(np.zeros(0, dtype=np.uint64), np.zeros(0, dtype=np.uint64)):
        for k in FIELDS:
            assert got[k] == 0, (k, got[k])
        assert got["hit_slots"] == [0] * 16


def test_noalloc_keeps_the_16_smallest_hits(engine):
    """More than 16 entries with q = 0, in shuffled order and spread over many CTAs: the hit
    list is the 16 smallest p in increasing order, the same on both calls."""
    rng = np.random.default_rng(11)
    n = 200000
    p = np.arange(3, 3 + 2 * n, 2, dtype=np.uint64)
    rng.shuffle(p)
    q = np.ones(n, dtype=np.uint64)
    zero = rng.choice(n, size=40, replace=False)
    q[zero] = 0
    want = sorted(int(x) for x in p[zero])[:16]
    a, b = _run_twice(p, q)
    for got in (a, b):
        assert got["nhits"] == 40
        assert got["hits"] == want
    assert a == b


def test_noalloc_refuses_oversized_input(engine):
    import mathpub_b200 as mp
    assert _noalloc(8, 8, mp.NOALLOC_MAX_COUNT + 1, 8, 0) == mp.MP_EINVAL
