"""Every form of the batched sieve the autotuner can pick gives the config-2 fixture exactly:
[1e15, 1e15 + 2^34) with per-2^24 block statistics and 2^20-integer segment hashes, for the
binned and the staged bucket scatter, each bucket threshold (the tile, half of it, a quarter of
it), and the persistent pipeline launch as well as the host loop of wave launches."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["pi", "twins", "max_gap", "gap_start", "tuple6", "tuple6_cks", "first_prime", "last_prime"]


@pytest.fixture(scope="module")
def eng():
    import mathpub_b200 as mp
    e = mp.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("staged,div,no_pipe", list(itertools.product([0, 1], [1, 2, 4], [0, 1])))
def test_config2_every_form(eng, configs, staged, div, no_pipe):
    import oracle
    c = configs["config2"]
    eng.tune_set(tile_log2=20, threads=1024, scatter_staged=staged, bucket_div=div, no_pipeline=no_pipe)
    r = eng.sieve_range(c["lo"], c["hi"], block_log2=c["block_log2"], hash_log2=c["hash_log2"])
    assert {k: r[k] for k in KEYS} == c["stats"]
    bl = r["blocks"]
    arr = np.ascontiguousarray(np.stack([bl[n] for n in bl.dtype.names], axis=1).reshape(-1))
    assert int(oracle.o().or_fnv1a64(arr.ctypes.data, arr.nbytes)) == c["blocks_fnv"]
    h = np.ascontiguousarray(r["hashes"])
    assert int(oracle.o().or_fnv1a64(h.ctypes.data, h.nbytes)) == c["hashes_fnv"]


def test_tune_set_rejects_bad_values(eng):
    import mathpub_b200 as mp
    for knob, v in [("tile_log2", 17), ("threads", 300), ("bucket_div", 3), ("no_pipeline", 2), ("bpsw_variant", 4)]:
        with pytest.raises(mp.MathpubError):
            eng.tune_set(**{knob: v})
    assert mp.lib().mp_tune_set(eng.handle, 99, 0) == mp.MP_EINVAL


def test_graph_replay_after_other_heights_and_forms(eng):
    """Batched calls replay a CUDA graph captured on an identical earlier call.  The graph
    reads the scatter's CTA bounds from device memory, so a call at another height (other
    bucket primes) or under another tuned form between two identical calls must not change
    what the replay computes.  Plain-mode calls never use graphs and give the answer."""
    import mathpub_b200 as mp
    eng.tune_set(tile_log2=20, threads=1024, scatter_staged=1, bucket_div=1, no_pipeline=1)
    ranges = [(10 ** 15, 10 ** 15 + (1 << 32)), (10 ** 12, 10 ** 12 + (1 << 32)), (10 ** 18, 10 ** 18 + (1 << 30))]
    want = {}
    for lo, hi in ranges:
        r = eng.sieve_range(lo, hi, mode=mp.MODE_PLAIN)
        want[lo] = {k: r[k] for k in KEYS}
    seq = [0, 0, 1, 1, 0, 2, 2, 1, 0, 2]
    for i in seq:
        lo, hi = ranges[i]
        r = eng.sieve_range(lo, hi)
        assert {k: r[k] for k in KEYS} == want[lo], (i, lo)
    # the same call under each form in turn, twice each (direct run, then replay)
    for staged, div in [(1, 2), (0, 1), (1, 4), (1, 1)]:
        eng.tune_set(scatter_staged=staged, bucket_div=div)
        for _ in range(2):
            r = eng.sieve_range(*ranges[0])
            assert {k: r[k] for k in KEYS} == want[ranges[0][0]], (staged, div)
