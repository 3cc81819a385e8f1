"""The allocation-free entry point mp_wieferich_stats_noalloc, called through the C ABI.

Some callers cannot allocate device memory (their framework's allocator owns the device,
or they run where a cudaMalloc, which can synchronise the device, is not allowed).  This
entry point serves them from a fixed scratch array inside the library.  Its results must
equal those of mp_wieferich_range on the same primes, call after call, because the scratch
that one call leaves behind must not leak into the next.

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
    return d


@pytest.mark.parametrize("lo,hi", [(1000, 4000), (10 ** 12, 10 ** 12 + 10 ** 7)])
def test_noalloc_matches_range_entry(engine, lo, hi):
    import torch
    import mathpub_b200 as mp
    want = engine.wieferich_range(lo, hi)
    p = engine.primes_range(lo, hi)
    q = engine.fermat_quotient(p)
    dev = torch.device("cuda", 0)
    d_p = torch.from_numpy(p.view(np.int64)).to(dev)
    d_q = torch.from_numpy(q.view(np.int64)).to(dev)
    s = torch.cuda.Stream(device=dev)
    for _ in range(2):                                     # two calls in a row
        stats = torch.full((7 + 16,), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(d_p.data_ptr(), d_q.data_ptr(), len(p), stats.data_ptr(), s.cuda_stream)
        assert rc == mp.MP_OK
        s.synchronize()
        got = _read(stats)
        for k in FIELDS:
            assert got[k] == want[k], (k, got[k], want[k])
        assert got["hits"] == want["hits"]


def test_noalloc_refuses_oversized_input(engine):
    import mathpub_b200 as mp
    assert _noalloc(8, 8, (1 << 24) + 1, 8, 0) == mp.MP_EINVAL
