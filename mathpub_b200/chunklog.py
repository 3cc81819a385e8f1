"""Chunk logs in the reference tools' own formats, computed on the GPU, so that a GPU run can be
checked by the reference CPU tools line by line (and resumed by them).

    python -m mathpub_b200.chunklog wieferich START END [-c CHUNK] [-L FILE]
    python -m mathpub_b200.chunklog twins N [-s CHUNK_NUMBERS] [-f FIRST] [-L FILE]

wieferich  The -L log of A001220/wieferich.c for base 2 (A001220/wieferich.c:1166-1171):
           "C <lo> <hi> <primes> 2:<checksum as 16 hex digits>" per chunk, chunk i =
           [START + i CHUNK, START + (i + 1) CHUNK), END rounded up to a chunk boundary
           (:1386-1392).  The checksum is the sum mod 2^64 of mix64(q XOR p 0x9E3779B97F4A7C15)
           over the tested primes (all odd primes), which is what the reference's dcheck.sh
           compares between a GPU run and the CPU tool.
twins      The -l log of A007508/a007508.c (:637, :874): "k <n> <idx> <chunk_k> <count>" per
           chunk of decade n and "d <n> <a(n)>" per finished decade.  Decade n covers the k
           in [K(n-1), K(n)), K(n) = (10^n - 10) / 30, where a twin pair (p, p + 2) with p > 5
           is attributed to k = p div 30 (:656-660, README "How it works"); chunk_k =
           CHUNK_NUMBERS / 30 (at least 64; default 10^max(9, n-4) / 30 capped at 10^13 / 30,
           :662-666).  The pairs (3, 5) and (5, 7) are added to decade 1, as the tool does.
"""
import argparse
import sys


def wieferich_lines(engine, start, end, chunk):
    """Lines of the base-2 Wieferich chunk log for [start, end) in chunks of `chunk`."""
    if end <= start or chunk <= 0:
        raise ValueError("need start < end and chunk > 0")
    nchunks = (end - start + chunk - 1) // chunk
    for i in range(nchunks):
        lo = start + i * chunk
        hi = lo + chunk
        w = engine.wieferich_range(lo, hi)
        yield f"C {lo} {hi} {w['primes']} 2:{w['cks']:016x}"


def kbound(n):
    return 0 if n < 1 else (10 ** n - 10) // 30


def default_chunk_k(n):
    e = min(max(n - 4, 9), 13)
    return 10 ** e // 30


def twin_lines(engine, n_max, chunk_numbers=0, first=1):
    """Lines of the A007508 chunk log for decades first..n_max (with their "d" lines)."""
    cumulative = 0
    for n in range(1, n_max + 1):
        k0, k1 = kbound(n - 1), kbound(n)
        ck = max(64, chunk_numbers // 30 if chunk_numbers else default_chunk_k(n))
        total = 0
        for i in range((k1 - k0 + ck - 1) // ck):
            klo = k0 + i * ck
            khi = min(klo + ck, k1)
            lo, hi = 30 * klo, 30 * khi
            c = engine.sieve_range(lo, hi)["twins"]
            c -= sum(1 for p in (3, 5) if lo <= p < hi)       # (3, 5), (5, 7) belong to decade 1
            total += c
            if n >= first:
                yield f"k {n} {i} {ck} {c}"
        cumulative += total + (2 if n == 1 else 0)
        if n >= first:
            yield f"d {n} {cumulative}"


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m mathpub_b200.chunklog")
    sub = ap.add_subparsers(dest="what", required=True)
    w = sub.add_parser("wieferich")
    w.add_argument("start", type=lambda s: int(float(s)) if "e" in s.lower() else int(s))
    w.add_argument("end", type=lambda s: int(float(s)) if "e" in s.lower() else int(s))
    w.add_argument("-c", "--chunk", type=int, default=10 ** 8)
    w.add_argument("-L", "--log")
    t = sub.add_parser("twins")
    t.add_argument("n", type=int)
    t.add_argument("-s", "--chunk-numbers", type=int, default=0)
    t.add_argument("-f", "--first", type=int, default=1)
    t.add_argument("-L", "--log")
    a = ap.parse_args(argv)
    import mathpub_b200 as mp
    e = mp.Engine(0)
    out = open(a.log, "a") if a.log else sys.stdout
    try:
        lines = wieferich_lines(e, a.start, a.end, a.chunk) if a.what == "wieferich" else \
            twin_lines(e, a.n, a.chunk_numbers, a.first)
        for line in lines:
            out.write(line + "\n")
            out.flush()
    finally:
        if out is not sys.stdout:
            out.close()
        e.close()


if __name__ == "__main__":
    main()
