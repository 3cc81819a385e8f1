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
