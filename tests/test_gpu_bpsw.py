"""BPSW on the GPU through the C ABI against the oracle: bit-exact verdicts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_small_and_edge_values(engine, orc):
    n = np.arange(0, 70000, dtype=np.uint64)
    assert np.array_equal(engine.bpsw(n), orc.bpsw(n))
    edges = np.array([2 ** 64 - 1 - k for k in range(0, 4000)] + [2 ** 63 + k for k in range(-2000, 2000)] +
                     [131 * 131, 131 * 131 - 2, 127 * 127, 2 ** 32 + 15, (2 ** 32 - 5) ** 2, 3 * 5 * 7 * 11],
                     dtype=np.uint64)
    assert np.array_equal(engine.bpsw(edges), orc.bpsw(edges))


def test_pseudoprimes(engine, ref_vectors):
    sp = np.array(ref_vectors["spsp2"] + ref_vectors["slpsp"], dtype=np.uint64)
    assert not engine.bpsw(sp).any()


def test_random_and_squares(engine, orc):
    rng = np.random.default_rng(3)
    xs = rng.integers(0, 2 ** 64 - 1, size=1 << 20, dtype=np.uint64) | np.uint64(1)
    r = rng.integers(2 ** 16, 2 ** 32 - 1, size=20000, dtype=np.uint64)
    sq = r * r
    pr = orc.primes_range(2 ** 31, 2 ** 31 + 2 ** 16).astype(np.uint64)
    psq = pr * pr
    allx = np.concatenate([xs, sq, psq])
    assert np.array_equal(engine.bpsw(allx), orc.bpsw(allx))


def test_batches_uneven_and_empty(engine, orc):
    import mathpub_b200 as mp
    n, lens = mp.bpsw_workload(99, 300000, 37)
    lens[5] = 0
    lens[6] += 0
    offs = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    lists = [n[offs[i]:offs[i] + lens[i]] for i in range(len(lens))] + [np.zeros(0, dtype=np.uint64),
                                                                       np.array([97], dtype=np.uint64)]
    got = engine.bpsw_batches(lists)
    for x, g in zip(lists, got):
        assert np.array_equal(g, orc.bpsw(x))


def test_plain_equals_batched_device_form(engine, orc):
    """The per-list launch form and the persistent work-queue form give the same bits."""
    import ctypes as C
    import torch
    import mathpub_b200 as mp
    n, lens = mp.bpsw_workload(5, 1 << 18, 64)
    pad = ((lens.astype(np.int64) + 31) // 32) * 32
    offs = np.concatenate([[0], np.cumsum(pad)]).astype(np.uint64)
    flat = np.zeros(int(offs[-1]), dtype=np.uint64)
    src = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    for i in range(len(lens)):
        flat[int(offs[i]):int(offs[i]) + int(lens[i])] = n[src[i]:src[i + 1]]
    dn = torch.from_numpy(flat.view(np.int64)).cuda()
    outs = []
    for mode in (mp.MODE_BATCHED, mp.MODE_PLAIN):
        db = torch.zeros(int(offs[-1]) // 32, dtype=torch.int32, device="cuda")
        rc = mp.lib().mp_bpsw_lists_dev(engine.handle, C.c_void_p(dn.data_ptr()), C.c_void_p(offs.ctypes.data),
                                        C.c_void_p(lens.ctypes.data), len(lens), C.c_void_p(db.data_ptr()), mode,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        outs.append(db.cpu().numpy().view(np.uint32))
    assert np.array_equal(outs[0], outs[1])
    want = orc.bpsw(n)
    for i in range(len(lens)):
        w = outs[0][int(offs[i]) // 32:(int(offs[i]) + int(pad[i])) // 32]
        bits = np.unpackbits(w.view(np.uint8), bitorder="little")[: int(lens[i])].astype(bool)
        assert np.array_equal(bits, want[src[i]:src[i + 1]])


def test_full_size_batch_matches_fixture(engine, configs):
    """The 2^26-candidate batch in 4096 uneven lists: verdict bytes hash as the oracle's and
    the reference's (tests/golden/configs.json)."""
    import mathpub_b200 as mp
    import oracle
    c3 = configs["config3"]
    n, lens = mp.bpsw_workload(c3["seed"], c3["count"], c3["nlists"])
    offs = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    got = engine.bpsw_batches([n[offs[i]:offs[i + 1]] for i in range(len(lens))])
    v = np.concatenate(got)
    assert int(v.sum()) == c3["primes"]
    packed = np.packbits(v, bitorder="little")
    assert int(oracle.o().or_fnv1a64(packed.ctypes.data, packed.nbytes)) == c3["verdict_fnv"]
