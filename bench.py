#!/usr/bin/env python
"""bench.py -- sieved integers/s at 1e15 (headline), u64 BPSW tests/s, batched vs plain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the large-offset sieve of [1e15, 1e15 + 2^34) on one GPU with every output of
that workload (per-2^24-block prime counts, twin counts, 6-tuple counts and checksums,
maximal gaps with their positions, per-2^20-integer FNV-1a hashes of the prime bitmap).
Under torchrun each rank sieves its own 2^34-integer range above 1e15 (weak scaling; the
ranges share nothing, so there is no collective in the data path; NCCL only carries the
barrier and the max-over-ranks of the device times).

Rank 0 prints one JSON line.  `value` = integers sieved by all ranks / the slowest rank's
summed device time of the K timed steps (CUDA events on the launching stream; L2 flushed
with a 256 MiB write between steps, outside the timed events).  `e2e` = the same workload
through the public host API mp_sieve_range (results copied back to host memory each step),
timed by the host clock.  The BPSW and plain-form numbers are reported beside it.

--impl reference: the CPU implementation of the same workload on this machine's cores (the
oracle's restatement of the reference's odd-only sieve, with every output), on a bounded
sample of the range per step; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sieved ints/s @1e15 and u64 BPSW tests/s, batched vs plain; p50/p99 latency"
LO = 10 ** 15
SPAN = 1 << 34
BLOCK_LOG2 = 24
HASH_LOG2 = 20
BPSW_SEED, BPSW_COUNT, BPSW_LISTS = 0x3C0FFEE, 1 << 26, 4096
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one tile-kernel launch (a wave
# of 1184 tiles at 1e15), from an ncu capture of that launch, taken while the bucket records
# were still on the wheel of 30 (1.006e9 a step; the wheel of 210 writes 8.63e8)
TILE_TRAFFIC_BYTES = 597.9e6 + 297.7e6
# the same for the persistent pipeline launch of one step (None until captured)
PIPE_TRAFFIC_BYTES = None
WORKLOAD = ("large-offset sieve [1e15, 1e15+2^34) per GPU, odd-only bitmap, sieving primes up to 31623048, "
            "wheel/pattern presieve 3..89, bucket sieve above the tile; outputs per-2^24-block pi, twins, "
            "6-tuples {0,4,6,10,12,16} with checksum, max gap + start, per-2^20 FNV-1a bitmap hashes")


def peaks_file():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as g:
            for line in g:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_work(primes, lo, hi, tile_bits, staged=True):
    """Exact marks of the sieve: the multiples m = k q of each sieving prime q >= 97 with
    max(lo, q^2) <= m < hi + tail, split at the tile size.  Primes q <= tile_bits mark the k
    coprime to 30 (the wheel of 30; the presieve patterns mark the multiples of 3 and 5) with
    shared-memory atomics; larger primes write a bucket record (4 bytes written + 4 read) for the
    k coprime to 210 (the staged scatter's wheel of 210: the patterns mark the multiples of 7 too);
    with the binned scatter (staged=False) the bucket primes keep the wheel of 30."""
    qi = primes[primes >= 97].astype(np.uint64)
    top = hi + (1 << 16)
    start = np.maximum(np.full(len(qi), lo, dtype=np.uint64), qi * qi)
    k0 = (start + qi - np.uint64(1)) // qi         # first k with k q >= start
    k1 = np.maximum((np.uint64(top) + qi - np.uint64(1)) // qi, k0)

    def coprime_below(k, wheel):                   # k' < k with gcd(k', wheel) = 1
        res = [r for r in range(wheel) if np.gcd(r, wheel) == 1]
        below = np.array([sum(1 for r in res if r < x) for x in range(wheel)], dtype=np.uint64)
        return np.uint64(len(res)) * (k // np.uint64(wheel)) + below[(k % np.uint64(wheel)).astype(np.int64)]

    small = qi <= np.uint64(tile_bits)
    wheel = 210 if staged else 30
    m30 = (coprime_below(k1[small], 30) - coprime_below(k0[small], 30)).astype(np.float64)
    mb = (coprime_below(k1[~small], wheel) - coprime_below(k0[~small], wheel)).astype(np.float64)
    return float(m30.sum()), float(mb.sum())


def _bitlen64(x):
    """bit length of each uint64 (0 for 0), exact: the two 32-bit halves go through float64"""
    x = np.asarray(x, dtype=np.uint64)
    hi = (x >> np.uint64(32)).astype(np.float64)
    lo = (x & np.uint64(0xffffffff)).astype(np.float64)
    bh = np.frexp(hi)[1].astype(np.int64)
    bl = np.frexp(lo)[1].astype(np.int64)
    return np.where(hi > 0, 32 + bh, bl)


def _odd_part(x):
    """x / 2^v2(x) for nonzero uint64 x"""
    x = np.asarray(x, dtype=np.uint64)
    low = x & (~x + np.uint64(1))
    return x >> (_bitlen64(low) - 1).astype(np.uint64)


TD_PRIMES = [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103,
             107, 109, 113, 127]
# 32-bit multiply or multiply-add instructions (the multiply pipe) in one Montgomery product:
# two limbs, 8 for the product, 4 for m = t n^-1 mod 2^64 and 7 for the high half of m n (the
# subtracting reduction, mp_mont64.cuh); three limbs of the Fermat kernel, three rows of
# 3 + 3 (a b_i) + 1 (m) + 3 + 3 (m N) (mp_fermat.cu)
IMAD_PER_PRODUCT_BPSW = 19
IMAD_PER_PRODUCT_FERMAT_K3 = 39


def bpsw_products(n, prime_mask):
    """Montgomery products of the BPSW kernels on the candidates n, counted exactly from the
    inputs: the base-2 ladder of every candidate that trial division leaves (bitlen(d) - 1
    squarings, n - 1 = d 2^s) and the Lucas ladder of every prime among them (bitlen(d') - 1
    steps, n + 1 = d' 2^s'; two products a step where Selfridge's D is 5, that is n = 2 or 3
    mod 5, four otherwise).  The squarings of the strong chains after the ladders and the set-up
    are left out, so this is a lower bound on the work."""
    n = np.asarray(n, dtype=np.uint64)
    surv = ((n & np.uint64(1)) == 1) & (n >= np.uint64(131 * 131))
    for q in TD_PRIMES:
        surv &= (n % np.uint64(q)) != 0
    ns = n[surv]
    sprp = int((_bitlen64(_odd_part(ns - np.uint64(1))) - 1).sum())
    npr = n[surv & prime_mask]
    npr = npr[npr != np.uint64(0xffffffffffffffff)]
    steps = _bitlen64(_odd_part(npr + np.uint64(1))) - 1
    m5 = npr % np.uint64(5)
    per = np.where((m5 == 2) | (m5 == 3), 2, 4)
    lucas = int((per * steps).sum())
    return sprp, lucas, int(surv.sum()), int(len(npr))


def run_ours(args):
    import torch
    import torch.distributed as dist
    import mathpub_b200 as mp
    from mathpub_b200 import shard

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and "RANK" in os.environ:
        pass
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    e = mp.Engine(local)
    L = mp.lib()
    # a stream of our own (the legacy default stream has handle 0, which the library reads
    # as "the handle's stream"); every launch and every timing event goes on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    lo, hi = shard.weak_shard(LO, SPAN, rank)
    nb = L.mp_sieve_nblocks(lo, hi, BLOCK_LOG2)
    nh = L.mp_sieve_nhashes(lo, hi, HASH_LOG2)
    d_out = torch.zeros(8, dtype=torch.int64, device=dev)
    d_blocks = torch.zeros(nb * 8, dtype=torch.int64, device=dev)
    d_hash = torch.zeros(nh, dtype=torch.int64, device=dev)
    import ctypes as C
    opts = mp.SieveOpts(mp.MODE_BATCHED, 0, BLOCK_LOG2, HASH_LOG2, 0)

    def sieve_dev(o=opts):
        rc = L.mp_sieve_range_dev(e.handle, lo, hi, C.byref(o), C.c_void_p(d_out.data_ptr()),
                                  C.c_void_p(d_blocks.data_ptr()), C.c_void_p(d_hash.data_ptr()), None,
                                  C.c_void_p(sp))
        if rc != 0:
            raise mp.MathpubError(rc, L.mp_last_error(e.handle).decode())

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(x):
        return shard.max_over_ranks(x, device=dev)

    # the measured autotuner picks the tile geometry at this height (and the Fermat variant)
    tune_report = e.autotune(LO) if args.autotune else "off"
    # warm-up (builds the prime tables and captures the graph on the first call)
    for _ in range(args.warmup):
        sieve_dev()
    barrier()

    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier()
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sieve_dev()
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    barrier()
    clocks = sampler.stop() if sampler else None
    tot_ms = max_over_ranks(sum(ms))
    value = world * args.steps * SPAN / (tot_ms / 1e3)

    # results of the timed steps (checked against the fixture when it is present)
    out = d_out.cpu().numpy().view(np.uint64)
    res = dict(zip(mp.STATS_FIELDS, [int(x) for x in out]))
    # whole-job statistics of [LO, LO + world SPAN): one all-gather of 8 words after timing
    res_job = shard.gather_join(res, "range", device=dev)

    # e2e through the host API: outputs copied to host memory every step
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.sieve_range(lo, hi, block_log2=BLOCK_LOG2, hash_log2=HASH_LOG2)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_tot = max_over_ranks(statistics.mean(e2e_ms))
    e2e_value = world * SPAN / (e2e_tot / 1e3)
    d2h = 64 + nb * 64 + nh * 8

    # profile pass: per-kernel device times on the launching stream
    e.profile(True)
    flush.zero_()
    sieve_dev()
    torch.cuda.synchronize()
    prof = e.profile_read()
    e.profile(False)
    tile_launches, tile_ms = prof["tile"]
    scat_launches, scat_ms = prof["scatter"]
    launches_per_step = sum(v[0] for v in prof.values())

    # plain (per-segment launch) form of the same workload, one step
    popts = mp.SieveOpts(mp.MODE_PLAIN, 0, BLOCK_LOG2, HASH_LOG2, 0)
    flush.zero_()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    sieve_dev(popts)
    b.record(stream)
    b.synchronize()
    plain_ms = max_over_ranks(a.elapsed_time(b))
    plain_out = dict(zip(mp.STATS_FIELDS, [int(x) for x in d_out.cpu().numpy().view(np.uint64)]))
    plain_value = world * SPAN / (plain_ms / 1e3)

    # BPSW: the seeded 2^26-candidate batch in 4096 uneven lists, device-resident
    n, lens = mp.bpsw_workload(BPSW_SEED + rank, BPSW_COUNT, BPSW_LISTS)
    pad = ((lens.astype(np.int64) + 31) // 32) * 32
    offs = np.concatenate([[0], np.cumsum(pad)]).astype(np.uint64)
    flat = np.zeros(int(offs[-1]), dtype=np.uint64)
    src = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    for i in range(len(lens)):
        flat[int(offs[i]):int(offs[i]) + int(lens[i])] = n[src[i]:src[i + 1]]
    dn = torch.from_numpy(flat.view(np.int64)).to(dev)
    db = torch.zeros(int(offs[-1]) // 32, dtype=torch.int32, device=dev)

    def bpsw_dev(mode):
        rc = L.mp_bpsw_lists_dev(e.handle, C.c_void_p(dn.data_ptr()), C.c_void_p(offs.ctypes.data),
                                 C.c_void_p(lens.ctypes.data), len(lens), C.c_void_p(db.data_ptr()), mode,
                                 C.c_void_p(sp))
        if rc != 0:
            raise mp.MathpubError(rc, L.mp_last_error(e.handle).decode())

    def time_bpsw(mode, steps):
        bpsw_dev(mode)
        torch.cuda.synchronize()
        tt = []
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bpsw_dev(mode)
            b.record(stream)
            b.synchronize()
            tt.append(a.elapsed_time(b))
        return max_over_ranks(statistics.mean(tt))

    bpsw_ms = time_bpsw(mp.MODE_BATCHED, max(3, args.steps))
    bpsw_bits = db.cpu().numpy().view(np.uint32).copy()
    bpsw_plain_ms = time_bpsw(mp.MODE_PLAIN, 2)
    plain_bits = db.cpu().numpy().view(np.uint32)
    bpsw_same = bool(np.array_equal(bpsw_bits, plain_bits))
    bpsw_primes = int(np.unpackbits(bpsw_bits.view(np.uint8)).sum())
    pmask = np.unpackbits(bpsw_bits.view(np.uint8), bitorder="little")[:len(flat)].astype(bool)
    sprp_products, lucas_products, bpsw_survivors, bpsw_lucas_n = bpsw_products(flat, pmask)

    peaks = e.probe_peaks()
    hbm, hbm_src = peaks_file()

    fermat = run_fermat(e, world, rank, dev, peaks["imad32"]) if not args.quick else None
    config1 = run_config1(e, dev, stream, flush, peaks, args.steps) if rank == 0 else None
    reference_gpu = run_reference_gpu() if (rank == 0 and world == 1 and not args.quick) else None
    chains = run_chains(e) if (rank == 0 and not args.quick) else None
    tuples = run_tuples(e) if (rank == 0 and not args.quick) else None
    serving = run_serving(e, args) if (rank == 0 and not args.quick and args.serve_requests) else None

    line = None
    if rank == 0:
        primes = e.primes_range(3, int(np.sqrt(float(hi + (1 << 16)))) + 2)
        tile_bits = 1 << 20
        import re
        m = re.search(r"sieve choice: tile 2\^(\d+)", tune_report)
        if m:
            tile_bits = 1 << int(m.group(1))
        m = re.search(r"bucket threshold tile/(\d+)", tune_report.split("sieve choice")[-1])
        bucket_div = int(m.group(1)) if m else 1
        ntiles = -(-((hi + (1 << 16) - lo) // 2) // tile_bits)
        staged = "binned scatter" not in tune_report.split("sieve choice")[-1]
        marks_small, marks_large = algorithmic_work(primes, lo, hi, tile_bits // bucket_div, staged)
        pipe_launches, pipe_ms = prof.get("pipeline", (0, 0.0))
        if pipe_launches:
            # one persistent launch per step runs the scatter and the tiles: its bytes are the
            # bucket records written and read back (4 B each way) and the bitmap written
            kname, klaunches, kms = "sieve_pipeline_kernel", pipe_launches, pipe_ms
            kbytes = (marks_large * 8 + ntiles * (tile_bits // 8)) / pipe_launches
            ktraffic = PIPE_TRAFFIC_BYTES
            knote = ("bytes = bucket records written and read (4 B each way per large-prime hit) + bitmap written; "
                     "the persistent launch also runs the scatter, so the atomic rate below is over the whole step")
        else:
            kname, klaunches, kms = f"tile_kernel<{tile_bits.bit_length() - 1},0>", tile_launches, tile_ms
            kbytes = (marks_large * 4 + ntiles * (tile_bits // 8)) / max(tile_launches, 1)
            ktraffic = TILE_TRAFFIC_BYTES
            knote = ("bytes = bucket records read (4 B per large-prime hit) + bitmap written; traffic = DRAM bytes of "
                     "one launch from an ncu capture taken with the bucket records on the wheel of 30 (14% more "
                     "records than this build's wheel of 210); the kernel is bound by instruction issue and "
                     "shared-memory atomics, see roofline_smem")
        tile_avg_s = kms / max(klaunches, 1) / 1e3
        achieved = kbytes / tile_avg_s / 1e9
        smem_marks_rate = (marks_small + marks_large) / (kms / 1e3)
        ref_fixture = None
        try:
            with open(os.path.join(ROOT, "tests", "golden", "configs.json")) as f:
                ref_fixture = json.load(f)["config2"]["stats"]
        except Exception:
            pass
        cpu = cpu_baseline() if world == 1 else None
        line = {
            "metric": METRIC, "value": value, "unit": "ints/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "lo": lo, "span": SPAN, "block_log2": BLOCK_LOG2,
                       "hash_log2": HASH_LOG2, "per_rank_range": "[1e15 + r 2^34, 1e15 + (r+1) 2^34)",
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world} (disjoint ranges)"},
            "e2e": {"value": e2e_value, "unit": "ints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                    "api": "mp_sieve_range (host buffers)"},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": ktraffic, "kernel": kname,
                         "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)" if hbm_src == "measured" else "fallback",
                         "algorithmic_bytes_per_launch": kbytes, "avg_launch_ms": tile_avg_s * 1e3,
                         "bucket_threshold": tile_bits // bucket_div, "note": knote},
            "roofline_smem": {"bound": "smem_atomics", "achieved": smem_marks_rate,
                              "peak": peaks["smem_atomic_conflict_free"], "unit": "atomic ops/s",
                              "frac": smem_marks_rate / peaks["smem_atomic_conflict_free"],
                              "peak_random_addresses": peaks["smem_atomic_random"],
                              "frac_of_random_peak": smem_marks_rate / peaks["smem_atomic_random"],
                              "marks_smem": marks_small, "marks_bucket": marks_large,
                              "peak_source": "measured in this run (mp_probe_peaks)"},
            "kernels_ms_per_step": {k: v[1] for k, v in prof.items() if v[0]},
            "plain": {"value": plain_value, "unit": "ints/s", "ms_per_step": plain_ms,
                      "batched_over_plain": value / plain_value, "same_results": plain_out == res},
            "bpsw": {"tests_per_s": world * BPSW_COUNT / (bpsw_ms / 1e3), "ms_per_batch": bpsw_ms,
                     "plain_tests_per_s": world * BPSW_COUNT / (bpsw_plain_ms / 1e3),
                     "plain_ms_per_batch": bpsw_plain_ms, "batched_over_plain": bpsw_plain_ms / bpsw_ms,
                     "same_verdicts": bpsw_same, "primes": bpsw_primes,
                     "roofline": imad_roofline((sprp_products + lucas_products) * IMAD_PER_PRODUCT_BPSW, bpsw_ms,
                                               peaks["imad32"], {
                         "products_base2_ladders": sprp_products, "products_lucas_ladders": lucas_products,
                         "candidates_past_trial_division": bpsw_survivors, "lucas_candidates": bpsw_lucas_n,
                         "imad_per_product": IMAD_PER_PRODUCT_BPSW,
                         "note": "achieved = Montgomery products counted exactly from the inputs (base-2 ladders of "
                                 "the trial-division survivors, Lucas ladders of the primes; chain squarings and "
                                 "set-up left out: a lower bound) x 32-bit multiply instructions per product / "
                                 "kernel time; peak = the 32-bit IMAD rate measured in this run"}),
                     "workload": "2^26 seeded odd u64 (60% uniform [2^40,2^64), 30% p*q near 2^62, "
                                 "10% (k+1)(2k+1) / Chernick), 4096 lists, log-uniform lengths"},
            "config1": config1,
            "reference_gpu": reference_gpu,
            "fermat": fermat,
            "chains": chains,
            "tuples": tuples,
            "serving": serving,
            "autotune": [s for s in tune_report.strip().splitlines() if "choice" in s] if tune_report != "off" else "off",
            "probes": peaks,
            "results": res, "results_job": res_job if world > 1 else None,
            "results_match_fixture": (res == ref_fixture) if (ref_fixture and rank == 0 and lo == LO) else None,
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    e.close()
    if line:
        print(json.dumps(line), flush=True)


C1_LO, C1_HI, C1_TILE_LOG2, C1_HASH_LOG2 = 10 ** 9, 11 * 10 ** 8, 18, 19


def run_config1(e, dev, stream, flush, peaks, steps):
    """Config 1: the plain segmented sieve of [1e9, 1.1e9) in 32 KiB segments (tiles of 2^18
    bits), sieving primes up to isqrt of the sieved top, outputs pi, twins, the widest gap with
    its start, 6-tuples and the FNV-1a hash of each 32 KiB segment's bitmap.  Device time with
    CUDA events on the launching stream, L2 flushed between steps; the same call in the plain
    form; marks per second of the dominant kernel against the shared-memory atomic rates."""
    import ast
    import ctypes as C
    import torch
    import mathpub_b200 as mp
    L = mp.lib()
    sp = stream.cuda_stream
    nh = L.mp_sieve_nhashes(C1_LO, C1_HI, C1_HASH_LOG2)
    d_out = torch.zeros(8, dtype=torch.int64, device=dev)
    d_hash = torch.zeros(nh, dtype=torch.int64, device=dev)

    def call(mode):
        o = mp.SieveOpts(mode, C1_TILE_LOG2, 0, C1_HASH_LOG2, 0)
        rc = L.mp_sieve_range_dev(e.handle, C1_LO, C1_HI, C.byref(o), C.c_void_p(d_out.data_ptr()), None,
                                  C.c_void_p(d_hash.data_ptr()), None, C.c_void_p(sp))
        if rc != 0:
            raise mp.MathpubError(rc, L.mp_last_error(e.handle).decode())

    def timed(mode, k):
        for _ in range(3):
            call(mode)
        torch.cuda.synchronize()
        tt = []
        for _ in range(k):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            call(mode)
            b.record(stream)
            b.synchronize()
            tt.append(a.elapsed_time(b))
        return statistics.mean(tt)

    ms = timed(mp.MODE_BATCHED, max(3, steps))
    res = dict(zip(mp.STATS_FIELDS, [int(x) for x in d_out.cpu().numpy().view(np.uint64)]))
    hashes = d_hash.cpu().numpy().view(np.uint64).copy()
    plain_ms = timed(mp.MODE_PLAIN, 3)
    plain_same = dict(zip(mp.STATS_FIELDS, [int(x) for x in d_out.cpu().numpy().view(np.uint64)])) == res and \
        np.array_equal(d_hash.cpu().numpy().view(np.uint64), hashes)
    e.profile(True)
    call(mp.MODE_BATCHED)
    torch.cuda.synchronize()
    prof = e.profile_read()
    e.profile(False)
    kern_ms = prof["tile"][1] + prof.get("pipeline", (0, 0.0))[1]
    primes = e.primes_range(3, int(np.sqrt(float(C1_HI + (1 << 16)))) + 2)
    m_small, m_large = algorithmic_work(primes, C1_LO, C1_HI, 1 << C1_TILE_LOG2)
    rate = (m_small + m_large) / (kern_ms / 1e3)
    fix = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "configs.json")) as f:
            c1 = json.load(f)["config1"]
        want = ast.literal_eval(c1["stats"]) if isinstance(c1["stats"], str) else c1["stats"]
        wh = ast.literal_eval(c1["hashes"]) if isinstance(c1["hashes"], str) else c1["hashes"]
        fix = all(res[k] == want[k] for k in want) and [int(x) for x in hashes] == [int(x) for x in wh]
    except Exception:
        pass
    span = C1_HI - C1_LO
    return {"workload": "plain segmented sieve [1e9, 1.1e9), 32 KiB segments (2^18-bit tiles), sieving primes to "
                        "isqrt(hi + tail); pi, twins, max gap + start, 6-tuples, per-32 KiB-segment FNV-1a hashes",
            "value": span / (ms / 1e3), "unit": "ints/s", "ms_per_call": ms, "l2": "flushed between calls",
            "plain": {"value": span / (plain_ms / 1e3), "ms_per_call": plain_ms, "batched_over_plain": plain_ms / ms,
                      "same_results": plain_same},
            "kernels_ms": {k: v[1] for k, v in prof.items() if v[0]},
            "roofline_smem": {"bound": "smem_atomics", "achieved": rate, "unit": "atomic ops/s",
                              "peak": peaks["smem_atomic_random"], "frac": rate / peaks["smem_atomic_random"],
                              "peak_conflict_free": peaks["smem_atomic_conflict_free"],
                              "marks": m_small + m_large, "kernel_ms": kern_ms,
                              "note": "marks = wheel-30 multiples of the sieving primes >= 97 counted exactly; "
                                      "peak = random-address shared atomicOr rate measured in this run"},
            "results": res, "results_match_fixture": fix}


def run_fermat(e, world, rank, dev, imad_peak):
    """Config 4: every prime in [1e12 + r 4e9, 1e12 + (r+1) 4e9) from the GPU sieve, base-2
    Fermat quotients with the full statistics; device time of the quotient and reduction
    kernels (events on the handle's stream), and the host-API call end to end."""
    lo = 10 ** 12 + rank * 4 * 10 ** 9
    hi = lo + 4 * 10 ** 9
    e.wieferich_range(lo, hi)                         # warm-up
    t0 = time.perf_counter()
    r = e.wieferich_range(lo, hi)
    wall = time.perf_counter() - t0
    kms = e.last_kernel_ms()
    from mathpub_b200 import shard
    job = shard.gather_join(r, "wieferich", device=dev) if world > 1 else None
    fix = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "configs.json")) as f:
            c4 = json.load(f)["config4"]
        fix = all(r[k] == c4[k] for k in ("primes", "tests", "near", "flt", "cks", "ordered_hash")) if lo == 10 ** 12 else None
    except Exception:
        pass
    # products per prime: one per bit of p - 1 (square and double folded into one product where
    # 8N < R) and the multiply that leaves Montgomery form; every p in the range has 40 bits
    products = r["tests"] * (40 + 1)
    roof = imad_roofline(products * IMAD_PER_PRODUCT_FERMAT_K3, kms, imad_peak, {
        "products": products, "imad_per_product": IMAD_PER_PRODUCT_FERMAT_K3,
        "note": "achieved = (bitlen(p - 1) + 1) three-limb Montgomery products per prime x 39 32-bit multiply "
                "instructions per product / time of the quotient and statistics kernels"})
    return {"workload": "base-2 Fermat quotients of every prime in [1e12, 1e12+4e9) (per rank), 3-limb Montgomery",
            "tests": r["tests"], "tests_per_s": r["tests"] / (kms / 1e3), "kernel_ms": kms, "roofline": roof,
            "e2e_tests_per_s": r["tests"] / wall, "e2e_ms": wall * 1e3, "near": r["near"], "flt": r["flt"],
            "cks": r["cks"], "results_match_fixture": fix,
            "job": {k: job[k] for k in ("primes", "tests", "near", "flt", "cks", "ordered_hash", "nhits")} if job else None}


CHAIN_A15 = 1397398433200922807          # A016045 a(15): 16 primes with gaps 2, 4, ..., 30
CHAIN_SPAN = 2 * 10 ** 16


def run_chains(e):
    """The constellation sieve (mp_chain_sieve): chains of 16 consecutive primes with gaps 2,
    4, ..., 30 in [a15 - 1e16, a15 + 1e16), a15 = A016045 a(15); wall time of the host call
    (it synchronises), after a warm-up call that builds the wheel and patterns for k = 16."""
    lo = CHAIN_A15 - CHAIN_SPAN // 2
    e.chain_sieve(lo, lo + 10 ** 13, 16)
    t0 = time.perf_counter()
    heads, lens = e.chain_sieve(lo, lo + CHAIN_SPAN, 16)
    wall = time.perf_counter() - t0
    found = [(int(h), int(n)) for h, n in zip(heads, lens)]
    return {"workload": "chains of >= 16 consecutive primes with gaps 2, 4, ..., 30 in [a15 - 1e16, a15 + 1e16), "
                        "a15 = A016045 a(15) = 1397398433200922807",
            "value": CHAIN_SPAN / wall, "unit": "integers/s", "ms": wall * 1e3, "chains": found,
            "finds_a15": (CHAIN_A15, 16) in found}


SEXTUPLET = [0, 4, 6, 10, 12, 16]


def run_tuples(e):
    """Prime sextuplets p + {0, 4, 6, 10, 12, 16} in [1e15, 1e15 + 2e12) by the constellation
    sieve (mp_tuple_count, admissible classes only), against the reference's window of that
    range (count and checksum); best of three host calls after a warm-up."""
    lo, hi = 10 ** 15, 10 ** 15 + 2 * 10 ** 12
    e.tuple_count(lo, lo + 10 ** 11, SEXTUPLET)
    best, res = None, None
    for _ in range(3):
        t0 = time.perf_counter()
        res = e.tuple_count(lo, hi, SEXTUPLET)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    fix = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "ref_vectors.json")) as f:
            w = json.load(f)["sext_windows"][0]
        fix = (w["lo"], w["hi"], w["count"], w["cks"]) == ("1e15", "1e15+2e12", res[0], res[1])
    except Exception:
        pass
    return {"workload": "prime sextuplets p + {0,4,6,10,12,16}, p in [1e15, 1e15+2e12)", "value": (hi - lo) / best,
            "unit": "integers/s", "ms": best * 1e3, "count": res[0], "cks": res[1], "matches_reference_window": fix}


def run_serving(e, args):
    """Config 5: a seeded stream of mixed requests arriving as a Poisson process.  70% range
    queries [lo, lo+len), lo log-uniform in [1e9, 1e18], len log-uniform in [2^16, 2^32]; 30%
    primality batches of 1..65536 candidates from the BPSW workload distribution.  The arrival
    rate is 70% of the capacity measured by a burst; latency = completion - submission (host
    clock).  Baseline: a sample of the same requests, each run alone with plain launches."""
    import threading
    import mathpub_b200 as mp
    import torch
    rng = np.random.default_rng(0x5E17E)
    pool, _ = mp.bpsw_workload(0x5E17E, 1 << 22, 0)

    def make(n):
        out = []
        for _ in range(n):
            if rng.random() < 0.7:
                lo = int(10 ** rng.uniform(9, 18))
                out.append(("r", lo, lo + int(2 ** rng.uniform(16, 32))))
            else:
                k = int(2 ** rng.uniform(0, 16))
                a = int(rng.integers(0, len(pool) - k))
                out.append(("b", pool[a:a + k]))
        return out

    def work(reqs):
        return (sum(r[2] - r[1] for r in reqs if r[0] == "r"), sum(len(r[1]) for r in reqs if r[0] == "b"))

    with mp.Server(e, streams=4) as srv:
        # capacity from a burst
        burst = make(3000)
        t0 = time.perf_counter()
        ids = [srv.submit_range(r[1], r[2]) if r[0] == "r" else srv.submit_bpsw(r[1]) for r in burst]
        for rid in ids:
            while srv.poll(rid, wait_ms=1000) is None:
                pass
        cap = len(burst) / (time.perf_counter() - t0)
        rate = 0.7 * cap
        reqs = make(args.serve_requests)
        arr = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        res = [None] * len(reqs)
        ids = [None] * len(reqs)
        ready = threading.Semaphore(0)

        def poller():
            for i in range(len(reqs)):
                ready.acquire()
                r = None
                while r is None:
                    r = srv.poll(ids[i], wait_ms=1000)
                res[i] = r

        th = threading.Thread(target=poller)
        th.start()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            d = arr[i] - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids[i] = srv.submit_range(r[1], r[2]) if r[0] == "r" else srv.submit_bpsw(r[1])
            ready.release()
        th.join()
        span = max(x["done_s"] for x in res) - min(x["submit_s"] for x in res)
        lat = np.array([x["done_s"] - x["submit_s"] for x in res]) * 1e3
        bad = sum(1 for x in res if x["status"] != 0)
    ints, tests = work(reqs)
    # each request alone with plain launches (a sample)
    sample = reqs[:60]
    L = mp.lib()
    alone = []
    for r in sample:
        t0 = time.perf_counter()
        if r[0] == "r":
            e.sieve_range(r[1], r[2], mode=mp.MODE_PLAIN)
        else:
            n = np.ascontiguousarray(r[1], dtype=np.uint64)
            pad = (len(n) + 31) // 32 * 32
            flat = np.zeros(pad, dtype=np.uint64)
            flat[:len(n)] = n
            dn = torch.from_numpy(flat.view(np.int64)).cuda()
            db = torch.zeros(pad // 32 + 1, dtype=torch.int32, device="cuda")
            offs = np.array([0, pad], dtype=np.uint64)
            lens = np.array([len(n)], dtype=np.uint32)
            import ctypes as C
            L.mp_bpsw_lists_dev(e.handle, C.c_void_p(dn.data_ptr()), C.c_void_p(offs.ctypes.data),
                                C.c_void_p(lens.ctypes.data), 1, C.c_void_p(db.data_ptr()), mp.MODE_PLAIN, None)
            torch.cuda.synchronize()
        alone.append(time.perf_counter() - t0)
    alone = np.array(alone) * 1e3
    return {"requests": len(reqs), "rate_req_per_s": rate, "burst_capacity_req_per_s": cap,
            "throughput_req_per_s": len(reqs) / span, "ints_per_s": ints / span, "tests_per_s": tests / span,
            "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
            "latency_ms_mean": float(lat.mean()), "failed": bad, "streams": 4,
            "alone_plain_sample": {"requests": len(sample), "req_per_s": len(sample) / (alone.sum() / 1e3),
                                   "latency_ms_p50": float(np.percentile(alone, 50)),
                                   "latency_ms_p99": float(np.percentile(alone, 99))},
            "served_over_alone_throughput": (len(reqs) / span) / (len(sample) / (alone.sum() / 1e3))}


REF_GPU_DIR = os.path.join(ROOT, "baseline", "_ref")


def run_reference_gpu():
    """The reference's own GPU programs, built unmodified from their sources for sm_100a into
    baseline/_ref (oracle/Makefile, target refgpu), timed by their own clocks on this GPU:
    a158939_cuda's sieve + gap scan over [1e15, 1e15+2e12), a350826_cuda's base-2 strong-test
    benchmark on 2^24 odd numbers near 1e18, and wieferich_cuda's base-2 Fermat quotients of the
    primes of [1e12, 1e12+4e9).  Each line is the program's own output."""
    import re
    progs = [
        ("a158939_sieve_gap_scan", ["a158939_cuda", "bench", "1000000000000000", "-d", "2000000000000", "-N"],
         r"bench: .*?: ([\d.]+) s, ([\d.e+]+) numbers/s", "numbers/s",
         "the reference's GPU sieve + gap scan (A158939/cuda/a158939_cuda.cu) over [1e15, 1e15+2e12)"),
        ("a350826_base2_sprp", ["a350826_cuda", "mrbench", "1000000000000000000", "16777216"],
         r"grid \d+: ([\d.]+) s, ([\d.e+]+) tests/s", "tests/s",
         "the reference's GPU base-2 strong probable-prime round (A350826/cuda/a350826_cuda.cu mrbench), 2^24 odd "
         "numbers near 1e18; one round per number, not a full BPSW verdict"),
        ("wieferich_base2", ["wieferich_cuda", "bench", "1000000000000", "-d", "4000000000", "-b", "2"],
         r"bench .*? in ([\d.]+) s", "tests/s",
         "the reference's GPU Fermat quotients (A001220/cuda/wieferich_cuda.cu), base 2, primes of [1e12, 1e12+4e9)"),
    ]
    out = {}
    for name, cmd, pat, unit, what in progs:
        exe = os.path.join(REF_GPU_DIR, cmd[0])
        if not os.path.exists(exe):
            out[name] = {"unavailable": f"{exe} not built (oracle/Makefile refgpu needs the reference tree)"}
            continue
        try:
            t0 = time.perf_counter()
            r = subprocess.run([exe] + cmd[1:], capture_output=True, text=True, timeout=180)
            wall = time.perf_counter() - t0
        except Exception as ex:
            out[name] = {"unavailable": f"did not finish: {ex}"}
            continue
        text = r.stdout + r.stderr
        rec = {"what": what, "rc": r.returncode, "wall_s": wall, "output": text.strip().splitlines()[-3:]}
        ms = re.findall(pat, text)
        if ms and name != "wieferich_base2":
            best = max(float(m[1]) for m in ms)
            rec.update({"value": best, "unit": unit, "seconds": float(ms[-1][0])})
        elif ms:
            tp = re.search(r"([\d.e+]+) tests/s", text)
            if tp:
                rec.update({"value": float(tp.group(1)), "unit": unit, "seconds": float(ms[-1])})
        out[name] = rec
    return out


def imad_roofline(imad_ops, kernel_ms, peak, extra):
    achieved = imad_ops / (kernel_ms / 1e3)
    out = {"bound": "imad", "achieved": achieved, "peak": peak, "unit": "IMAD ops/s", "frac": achieved / peak,
           "traffic": None, "peak_source": "measured in this run (mp_probe_peaks imad32)"}
    out.update(extra)
    return out


def reference_twin_sieve(lo, hi, t):
    """The reference's own CPU sieve for one output of this workload: A007508's twin-class bucket
    sieve (count_twins_twin, A007508/a007508.c:514, built from its source into oracle/_ref) on the
    same sample, rounded to multiples of 30.  It sieves 3 of every 15 odd residues (twin classes
    only), so its integers/s is for the twin count alone."""
    import oracle
    if not oracle.have_ref_twins():
        return None
    a, b = -(-lo // 30) * 30, (hi // 30) * 30
    t0 = time.perf_counter()
    n = oracle.ref_twins(a, b, t)
    dt = time.perf_counter() - t0
    return {"value": (b - a) / dt, "unit": "ints/s", "cores": t, "kind": "reference", "twins": n,
            "sample": f"twin pairs in [{a}, {b}) by A007508/a007508.c count_twins_twin, {t} threads, {dt:.3f} s "
                      "(twin count only)"}


def cpu_baseline(sample_log2=31):
    """The oracle's restatement of the reference's odd-only sieve (every output of the
    workload) on [1e15, 1e15 + 2^31) with all host threads."""
    import oracle
    t = oracle.threads()
    lo, hi = LO, LO + (1 << sample_log2)
    t0 = time.perf_counter()
    oracle.sieve_range(lo, hi, block_log2=BLOCK_LOG2, hash_log2=HASH_LOG2, nthreads=t)
    dt = time.perf_counter() - t0
    out = {"value": (hi - lo) / dt, "unit": "ints/s", "cores": t, "kind": "port",
           "sample": f"[1e15, 1e15+2^{sample_log2}) with every output, {t} threads, {dt:.2f} s"}
    tw = reference_twin_sieve(lo, hi, t)
    if tw:
        out["reference_twin_sieve"] = tw
    if oracle.have_ref():
        import mathpub_b200 as mp
        n, _ = mp.bpsw_workload(BPSW_SEED, 1 << 22, 0)
        t0 = time.perf_counter()
        oracle.ref_bpsw(n, t)
        dt = time.perf_counter() - t0
        out["bpsw"] = {"value": len(n) / dt, "unit": "tests/s", "cores": t, "kind": "reference",
                       "sample": f"2^22 candidates of the BPSW workload, reference sprp2_64x4 + slprp64, {t} threads"}
        p = oracle.primes_range(10 ** 12, 10 ** 12 + 4 * 10 ** 7, t)
        t0 = time.perf_counter()
        oracle.ref_fermat_q(p, t)
        dt = time.perf_counter() - t0
        out["fermat"] = {"value": len(p) / dt, "unit": "tests/s", "cores": t, "kind": "reference",
                         "sample": f"{len(p)} primes of [1e12, 1e12+4e7), reference run_group (8 lanes), {t} threads"}
        t0 = time.perf_counter()
        oracle.ref_count_sext(lo, hi, t)
        dt = time.perf_counter() - t0
        gs = os.path.join(ROOT, "oracle", "_ref", "gapsieve_cpu")
        if os.path.exists(gs):
            clo = CHAIN_A15 - 10 ** 14
            t0 = time.perf_counter()
            r = subprocess.run([gs, "-l", "16", "-s", str(clo), "-e", str(clo + 2 * 10 ** 14 - 1), "-q",
                                "-t", str(t)], capture_output=True, text=True)
            dt = time.perf_counter() - t0
            if r.returncode == 0:
                out["chains"] = {"value": 2e14 / dt, "unit": "integers/s", "cores": t, "kind": "reference",
                                 "sample": f"gapchain/gapsieve.c (its CPU build) -l 16 over [a15 - 1e14, a15 + 1e14), "
                                           f"{t} threads, {dt:.2f} s"}
        out["reference_sextuplet_count"] = {"value": (hi - lo) / dt, "unit": "ints/s", "kind": "reference",
                                            "sample": f"a350826 count [1e15, 1e15+2^{sample_log2}), {t} threads "
                                                      "(6-tuples only: it sieves the admissible classes, not all "
                                                      "integers)"}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    t = oracle.threads()
    sample = 1 << 31
    for _ in range(args.warmup if args.warmup < 2 else 1):
        oracle.sieve_range(LO, LO + (1 << 26), block_log2=BLOCK_LOG2, hash_log2=HASH_LOG2, nthreads=t)
    times = []
    for k in range(args.steps):
        lo = LO + k * sample
        t0 = time.perf_counter()
        oracle.sieve_range(lo, lo + sample, block_log2=BLOCK_LOG2, hash_log2=HASH_LOG2, nthreads=t)
        times.append(time.perf_counter() - t0)
    value = sample * len(times) / sum(times)
    tw = reference_twin_sieve(LO, LO + sample, t)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "ints/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_per_step": "2^31 integers of the range, every output"},
            "cpu_baseline": {"value": value, "unit": "ints/s", "cores": t, "kind": "port",
                             "sample": f"[1e15 + k 2^31, +2^31) per step, {t} threads; the reference has no CPU "
                                       "function that sieves a range with these outputs (its odd-only sieve in "
                                       "A228768/a228768.c:372-415 runs an emirp test on every prime), so the "
                                       "oracle's restatement of that sieve with every output is timed; the "
                                       "reference's own twin-class sieve is timed beside it "
                                       "(reference_twin_sieve)"},
            "e2e": {"value": value, "unit": "ints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if tw:
        line["reference_twin_sieve"] = tw
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--serve-requests", type=int, default=100000)
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--quick", action="store_true", help="headline sieve, plain form and BPSW only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
