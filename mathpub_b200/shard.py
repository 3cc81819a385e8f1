"""Sharding a range over ranks (one process per GPU) and joining the ranks' statistics.

The reference tools split their work into independent chunks -- a range [lo, hi) per job --
and compare the per-chunk log lines afterwards (A001220/wieferich.c:1129-1177 writes one line
per chunk, A350826's run_quiet counts one window per call).  Across GPUs the same holds:
every rank sieves its own contiguous shard with no data-path exchange, and the only
collective is one all-gather of a few 64-bit statistics at the end, folded in rank order.

The statistics of include/mathpub_gpu.h are attributed to the prime that starts a pattern
(a gap belongs to the prime before it, a twin pair or 6-tuple to its first member), and each
rank sieves the tail past its shard, so the join of two adjacent shards is exact:
    pi, twins, tuple6                  add
    tuple6_cks                         add mod 2^64
    max_gap / gap_start                larger gap; a tie keeps the smaller start
    first_prime / last_prime           first of the left non-empty shard / last of the right
For the Wieferich statistics (A001220/wieferich.c:1051-1075) counts and the checksum add,
the ordered hash H <- H * 0x100000001b3 + mix64(p ^ mix64(q)) over the hashed terms of the
right shard joins as H_L * B^(terms_R) + H_R with terms = tests - flt, and the hit lists
concatenate (16 kept).
"""
import numpy as np

M64 = (1 << 64) - 1
FNV_PRIME = 0x100000001b3
STATS_FIELDS = ["pi", "twins", "max_gap", "gap_start", "tuple6", "tuple6_cks", "first_prime", "last_prime"]
WIEF_FIELDS = ["primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits"]
WIEF_HITS = 16


def split_range(lo, hi, world, align=1 << 24):
    """Contiguous shards [lo_r, hi_r) of [lo, hi), one per rank, in rank order.

    Interior cut points lie at lo + k * align, so per-block statistics (blocks of 2^block_log2
    integers from lo) and per-segment hashes (segments of 2^hash_log2 integers from lo & ~1)
    of the shards concatenate into those of the whole range when align is a multiple of both
    widths.  Shards differ in length by at most one align unit; trailing shards may be empty
    when the range holds fewer units than ranks."""
    if hi < lo or world < 1 or align < 2 or align & 1:
        raise ValueError("split_range: need lo <= hi, world >= 1 and an even align >= 2")
    units = -(-(hi - lo) // align)
    cuts = [lo + min(hi - lo, (units * r // world) * align) for r in range(world)] + [hi]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def weak_shard(lo, span, rank):
    """Weak scaling: rank r owns [lo + r span, lo + (r + 1) span)."""
    return lo + rank * span, lo + (rank + 1) * span


def join_range_stats(a, b):
    """Ordered join of the range statistics of [x, y) (a) and [y, z) (b)."""
    if not a["pi"]:
        return dict(b)
    if not b["pi"]:
        return dict(a)
    r = {"pi": a["pi"] + b["pi"], "twins": a["twins"] + b["twins"], "tuple6": a["tuple6"] + b["tuple6"],
         "tuple6_cks": (a["tuple6_cks"] + b["tuple6_cks"]) & M64,
         "first_prime": a["first_prime"], "last_prime": b["last_prime"]}
    if b["max_gap"] > a["max_gap"]:
        r["max_gap"], r["gap_start"] = b["max_gap"], b["gap_start"]
    else:
        r["max_gap"], r["gap_start"] = a["max_gap"], a["gap_start"]
    return r


def join_wief_stats(a, b):
    """Ordered join of the Wieferich statistics of two adjacent prime ranges."""
    r = {k: (a[k] + b[k]) & M64 for k in ("primes", "tests", "near", "flt", "cks", "nhits")}
    terms = (b["tests"] - b["flt"]) & M64
    r["ordered_hash"] = (a["ordered_hash"] * pow(FNV_PRIME, terms, 1 << 64) + b["ordered_hash"]) & M64
    r["hits"] = (list(a.get("hits", [])) + list(b.get("hits", [])))[:WIEF_HITS]
    return r


def fold(parts, join):
    """Join a list of per-shard statistics in shard order (the join is associative)."""
    acc = parts[0]
    for p in parts[1:]:
        acc = join(acc, p)
    return acc


def _pack(d, fields, extra=0):
    v = [d[k] & M64 for k in fields]
    if extra:
        h = list(d.get("hits", []))[:extra]
        v += h + [0] * (extra - len(h))
    return np.array(v, dtype=np.uint64).view(np.int64)


def _unpack(a, fields, extra=0):
    u = a.view(np.uint64)
    d = {k: int(u[i]) for i, k in enumerate(fields)}
    if extra:
        d["hits"] = [int(x) for x in u[len(fields):len(fields) + min(extra, d["nhits"])]]
    return d


def gather_join(stats, kind="range", device=None, group=None):
    """All-gather one rank's statistics (a dict) and return the join over all ranks in rank
    order, the same on every rank.  kind is "range" (mp_range_stats) or "wieferich"
    (mp_wief_stats).  device is where the gathered tensor lives: "cpu" for gloo, the rank's
    cuda device for nccl.  Without an initialised process group this returns the input."""
    import torch
    import torch.distributed as dist
    fields, extra, join = ((STATS_FIELDS, 0, join_range_stats) if kind == "range"
                           else (WIEF_FIELDS, WIEF_HITS, join_wief_stats))
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return dict(stats)
    world = dist.get_world_size(group)
    mine = torch.from_numpy(_pack(stats, fields, extra)).to(device or "cpu")
    bufs = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(bufs, mine, group=group)
    parts = [_unpack(t.cpu().numpy(), fields, extra) for t in bufs]
    return fold(parts, join)


def max_over_ranks(x, device=None, group=None):
    """The largest of one float per rank (device times of a step are reported as the max)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
