"""Host logic of the multi-rank path (CPU): range shards, the ordered join of per-shard
statistics, and the all-gather over a world_size-2 gloo group.  The per-shard numbers come
from the oracle, so the join is checked against the oracle run over the whole range."""
import json
import os
import socket

import numpy as np
import pytest

import oracle
from mathpub_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_split_range_properties():
    for lo, hi, world, align in [(0, 1000, 3, 8), (10**12 + 1, 10**12 + 1 + 5 * 2**20, 4, 2**20),
                                 (7, 7, 2, 2), (100, 130, 8, 16), (2**63, 2**63 + 2**40 + 6, 8, 2**24)]:
        parts = shard.split_range(lo, hi, world, align)
        assert len(parts) == world
        assert parts[0][0] == lo and parts[-1][1] == hi
        for (a, b), (c, d) in zip(parts, parts[1:]):
            assert b == c and a <= b
        for a, b in parts[:-1]:
            assert (b - lo) % align == 0 or b == hi
        lens = [b - a for a, b in parts if b - a]
        assert not lens or max(lens) - min(lens) <= align
    with pytest.raises(ValueError):
        shard.split_range(5, 4, 2)
    with pytest.raises(ValueError):
        shard.split_range(0, 10, 2, 3)
    assert shard.weak_shard(10**15, 2**34, 3) == (10**15 + 3 * 2**34, 10**15 + 4 * 2**34)


@pytest.mark.parametrize("lo,hi,world", [(10**9, 10**9 + 2**22, 2), (10**12 + 1, 10**12 + 1 + 3 * 2**20, 5),
                                         (1, 2**21, 3), (2**40 - 2**20, 2**40 + 2**20, 4)])
def test_join_of_shards_equals_whole(lo, hi, world):
    whole = oracle.sieve_range(lo, hi, block_log2=16, hash_log2=16)
    parts = shard.split_range(lo, hi, world, 1 << 16)
    got = [oracle.sieve_range(a, b, block_log2=16, hash_log2=16) for a, b in parts if b > a]
    joined = shard.fold([{k: g[k] for k in shard.STATS_FIELDS} for g in got], shard.join_range_stats)
    assert joined == {k: whole[k] for k in shard.STATS_FIELDS}
    # blocks and hashes of aligned shards concatenate into those of the whole range
    assert np.array_equal(np.concatenate([g["blocks"] for g in got]), whole["blocks"])
    assert np.array_equal(np.concatenate([g["hashes"] for g in got]), whole["hashes"])


def test_join_handles_empty_and_tied_shards():
    e = {k: 0 for k in shard.STATS_FIELDS}
    a = oracle.sieve_range(24, 28)            # no primes
    assert a["pi"] == 0
    b = oracle.sieve_range(29, 40)
    assert shard.join_range_stats({k: a[k] for k in e}, {k: b[k] for k in e}) == {k: b[k] for k in e}
    assert shard.join_range_stats({k: b[k] for k in e}, e) == {k: b[k] for k in e}
    # a tie on the largest gap keeps the earlier start
    left = dict(b, max_gap=6, gap_start=31)
    right = dict(b, max_gap=6, gap_start=97)
    assert shard.join_range_stats(left, right)["gap_start"] == 31


@pytest.mark.parametrize("lo,hi,world", [(1000, 200000, 2), (10**9, 10**9 + 3 * 10**6, 3)])
def test_wieferich_join_equals_whole(lo, hi, world):
    whole = oracle.wieferich_range(lo, hi)
    parts = shard.split_range(lo, hi, world, 2)
    got = [oracle.wieferich_range(a, b) for a, b in parts if b > a]
    assert shard.fold(got, shard.join_wief_stats) == whole


def _rank_main(rank, world, port, lo, hi, outdir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        a, b = shard.split_range(lo, hi, world, 1 << 16)[rank]
        mine = oracle.sieve_range(a, b, nthreads=2)
        joined = shard.gather_join({k: mine[k] for k in shard.STATS_FIELDS}, "range")
        wa, wb = shard.split_range(10**6, 10**6 + 4 * 10**5, world, 2)[rank]
        wj = shard.gather_join(oracle.wieferich_range(wa, wb, nthreads=2), "wieferich")
        slowest = shard.max_over_ranks(1.5 + rank)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"range": joined, "wief": wj, "max": slowest}, f)
    finally:
        dist.destroy_process_group()


def test_gloo_world2_gather_join(tmp_path):
    import torch.multiprocessing as tmp
    lo, hi, world = 10**10, 10**10 + 2**22, 2
    tmp.start_processes(_rank_main, args=(world, _free_port(), lo, hi, str(tmp_path)), nprocs=world,
                        join=True, start_method="spawn")
    whole = oracle.sieve_range(lo, hi)
    wwhole = oracle.wieferich_range(10**6, 10**6 + 4 * 10**5)
    for r in range(world):
        with open(tmp_path / f"rank{r}.json") as f:
            got = json.load(f)
        assert got["range"] == {k: whole[k] for k in shard.STATS_FIELDS}
        assert got["wief"] == wwhole
        assert got["max"] == 1.5 + world - 1
