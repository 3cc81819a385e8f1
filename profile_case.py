"""Run one workload between cudaProfilerStart/Stop, for `ncu --profile-from-start off`.

    python profile_case.py sieve  [--lo 1e15] [--log2span 32] [--tile 20] [--threads 1024]
    python profile_case.py bpsw   [--log2count 22]
    python profile_case.py fermat [--lo 1e12] [--span 1e8]
    python profile_case.py chain  [--lo 1e15] [--span 1e8] [--k 16] [--dec]

The tables are built and every kernel runs once before the profiled region, so the capture
holds only the steady-state launches of one call.
"""
import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import mathpub_b200 as mp  # noqa: E402


def num(s):
    return int(float(s)) if "e" in s.lower() else int(s)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["sieve", "bpsw", "fermat", "chain"])
    ap.add_argument("--lo", default="1e15")
    ap.add_argument("--log2span", type=int, default=32)
    ap.add_argument("--span", default="1e8")
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--log2count", type=int, default=22)
    ap.add_argument("--plain", action="store_true")
    ap.add_argument("--k", type=int, default=16)
    ap.add_argument("--dec", action="store_true")
    a = ap.parse_args()
    import torch
    e = mp.Engine(0)
    mode = mp.MODE_PLAIN if a.plain else mp.MODE_BATCHED
    if a.what == "sieve":
        lo = num(a.lo)
        hi = lo + (1 << a.log2span)
        run = lambda: e.sieve_range(lo, hi, block_log2=24, hash_log2=20, mode=mode, tile_log2=a.tile,
                                    threads=a.threads)
    elif a.what == "bpsw":
        n, _ = mp.bpsw_workload(0x3C0FFEE, 1 << a.log2count, 0)
        run = lambda: e.bpsw(n)
    elif a.what == "fermat":
        lo = num(a.lo)
        run = lambda: e.wieferich_range(lo, lo + num(a.span))
    else:
        lo = num(a.lo)
        run = lambda: e.chain_sieve(lo, lo + num(a.span), a.k, dec=a.dec)
    r0 = run()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    r1 = run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    if a.what == "bpsw":
        assert np.array_equal(r0, r1)
        print("primes", int(r1.sum()))
    elif a.what == "chain":
        assert all(np.array_equal(x, y) for x, y in zip(r0, r1))
        print("chains", len(r1[0]), [(int(h), int(n)) for h, n in zip(*r1)][:8])
    else:
        same = {k: r0[k] for k in r0 if not isinstance(r0[k], np.ndarray)} == \
               {k: r1[k] for k in r1 if not isinstance(r1[k], np.ndarray)}
        assert same
        print({k: v for k, v in r1.items() if not isinstance(v, np.ndarray)})
    e.close()


if __name__ == "__main__":
    main()
