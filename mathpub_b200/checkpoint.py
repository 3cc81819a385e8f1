"""Checkpoint files in the reference tools' own formats, computed on the GPU, so that a scan
started here can be finished (resumed) by the reference's CPU tool, and the other way round.

    python -m mathpub_b200.checkpoint wieferich START END FRONTIER [-c CHUNK] [-S FILE]

wieferich  The -S state of A001220/wieferich.c for base 2 (save_state / load_state,
           A001220/wieferich.c:1223-1320): "wieferich checkpoint 1", then "bases 2", "start",
           "chunk", "end" (END rounded up to a chunk boundary, :1386-1392), "frontier" (the
           number of finished chunks), the totals "primes", "tests", "near", "flt" over the
           finished chunks, "cks 2 <16 hex digits>", one "hit 2 <p> <chunk>" per solution
           below the frontier, and "end".  Chunk i is [START + i CHUNK, START + (i+1) CHUNK).
           `near` is the count of |A| <= T for the tool's -n T; without -n (T = 0, the
           tool's default) it is 0, and that is the only threshold written here.
           Running `wieferich scan START END -b 2 -c CHUNK -S FILE` on such a file resumes at
           the frontier and ends with the same summary and state as a scan that ran alone.

The twin tool (A007508/a007508.c) resumes from its chunk log (-l), which chunklog.py
writes.  The sextuplet tool's state (A350826/a350826.c:1756) counts chunks of its own
wheel classes and carries its own sieve's survivor and candidate counters, which a
different sieve cannot reproduce, so that state is not written.
"""
import argparse
import os
import sys


def wieferich_state(engine, start, end, chunk, frontier):
    """Text of the base-2 Wieferich checkpoint after the first `frontier` chunks of
    [start, end) in chunks of `chunk`, from engine.wieferich_range per chunk."""
    if end <= start or chunk <= 0:
        raise ValueError("need start < end and chunk > 0")
    nchunks = (end - start + chunk - 1) // chunk
    if not 0 <= frontier <= nchunks:
        raise ValueError(f"frontier must be in [0, {nchunks}]")
    primes = tests = flt = cks = 0
    hits = []
    for i in range(frontier):
        lo = start + i * chunk
        w = engine.wieferich_range(lo, lo + chunk)
        primes += w["primes"]
        tests += w["tests"]
        flt += w["flt"]
        cks = (cks + w["cks"]) % (1 << 64)
        hits += [(p, i) for p in w["hits"]]
    lines = ["wieferich checkpoint 1", "bases 2", f"start {start}", f"chunk {chunk}",
             f"end {start + nchunks * chunk}", f"frontier {frontier}", f"primes {primes}", f"tests {tests}",
             "near 0", f"flt {flt}", f"cks 2 {cks:016x}"]
    lines += [f"hit 2 {p} {c}" for p, c in hits]
    lines.append("end")
    return "\n".join(lines) + "\n"


def write_atomically(path, text):
    """Write to path.tmp and rename over path, as the reference does, so a crash never leaves a
    half-written checkpoint."""
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(text)
    os.replace(tmp, path)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m mathpub_b200.checkpoint")
    sub = ap.add_subparsers(dest="what", required=True)
    w = sub.add_parser("wieferich")
    w.add_argument("start", type=lambda s: int(float(s)) if "e" in s.lower() else int(s))
    w.add_argument("end", type=lambda s: int(float(s)) if "e" in s.lower() else int(s))
    w.add_argument("frontier", type=int)
    w.add_argument("-c", "--chunk", type=int, default=10 ** 9)
    w.add_argument("-S", "--state", default=None)
    a = ap.parse_args(argv)
    import mathpub_b200 as mp
    e = mp.Engine(0)
    try:
        text = wieferich_state(e, a.start, a.end, a.chunk, a.frontier)
    finally:
        e.close()
    if a.state:
        write_atomically(a.state, text)
    else:
        sys.stdout.write(text)


if __name__ == "__main__":
    main()
