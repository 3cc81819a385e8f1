"""Generate the golden fixtures in tests/golden/ (run where the reference tree exists).

    python tests/golden/make_golden.py [--skip-full]

ref_vectors.json   known answers held by the reference's own sources, extracted here by
                   pattern from the files (pseudoprime lists and sextuplet windows of
                   A350826/a350826.c, pi tables and windows of A158939/cuda/a158939_cuda.cu,
                   pi(1e9) of A001220/wieferich.c, twin counts of A007508/README.md, the
                   base-2 Wieferich primes of A001220/wieferich.c, the known terms of
                   A158939 (A158939/a158939.c:7-10) and A252768 (A252768/a252768.c:8-9), and the
                   A016045 table of gapchain/README.md (first heads of chains of gaps 2, 4, 6, ...),
                   its A263049 table (the first starts of the exact patterns of gaps ..., 6, 4, 2))
verify_py.json     windows computed by the reference's independent Python verifiers
                   (A001220/verify_wieferich.py, A350826/verify_a350826.py) run here
configs.json       the full-size workloads computed by the oracle (tests/ checks the oracle
                   against the two files above) and, where the reference's C builds, by
                   the reference itself; the two must agree or generation stops
"""
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
# the reference tree: $MATHPUB_REFERENCE, else its checkout on the machine that made the fixtures
REF = os.environ.get("MATHPUB_REFERENCE", "/root/reference")

import oracle  # noqa: E402

FNV_OFF, FNV_PRIME, M64 = 0xcbf29ce484222325, 0x100000001b3, (1 << 64) - 1


def fnv_bytes(b):
    """FNV-1a-64 of a byte string (computed by the oracle's C routine)."""
    a = np.frombuffer(bytes(b), dtype=np.uint8)
    return int(oracle.o().or_fnv1a64(a.ctypes.data, len(a)))


def fnv_u64s(a):
    """FNV-1a-64 over the little-endian bytes of a uint64 array (fast path via numpy)."""
    return fnv_bytes(np.ascontiguousarray(a, dtype="<u8").tobytes())


def src(path):
    with open(os.path.join(REF, path)) as f:
        return f.read()


def ints_in(block):
    return [int(x.rstrip("ULul")) for x in re.findall(r"\b\d+(?:ULL|UL|U|ull)?\b", block)]


def ref_vectors():
    a = src("A350826/a350826.c")
    out = {}
    m = re.search(r"static const u64 spsp2\[\] = \{(.*?)\};", a, re.S)
    out["spsp2"] = ints_in(m.group(1))
    m = re.search(r"static const u64 slpsp\[\] = \{(.*?)\};", a, re.S)
    out["slpsp"] = ints_in(m.group(1))
    m = re.search(r"static const u64 A350826\[\] = \{(.*?)\};", a, re.S)
    out["A350826"] = ints_in(m.group(1))
    m = re.search(r"static const window_t WINDOWS\[\] = \{(.*?)\{NULL", a, re.S)
    out["sext_windows"] = [
        {"lo": lo, "hi": hi, "count": int(c), "cks": int(k, 16)}
        for lo, hi, c, k in re.findall(r'\{"([^"]+)", "([^"]+)", (\d+), 0x([0-9a-fA-F]+)ULL\}', m.group(1))]
    g = src("A158939/cuda/a158939_cuda.cu")
    m = re.search(r"static const u64 PI10\[17\] = \{(.*?)\};", g, re.S)
    pi10 = ints_in(m.group(1))
    out["pi10"] = {str(k): v for k, v in enumerate(pi10) if v}
    out["pi_windows"] = []
    for m in re.finditer(r"run_scan\((\d+)ULL, (\d+)ULL,", g):
        want = re.search(r"S\.primes == (\d+)ULL", g[m.end():m.end() + 600])
        if want:
            out["pi_windows"].append({"lo": int(m.group(1)), "hi": int(m.group(2)), "pi": int(want.group(1))})
    m = re.search(r"run_scan\(0, 100000000000ULL.*?S\.primes == (\d+)ULL", g, re.S)
    out["pi_windows"].insert(0, {"lo": 0, "hi": 10 ** 11, "pi": int(m.group(1))})
    w = src("A001220/wieferich.c")
    m = re.search(r"S\.primes == (\d+)ULL", w)
    out["pi_1e9"] = int(m.group(1))
    m = re.search(r"\{ 2, 2, \{(\d+), (\d+)\}\}", w)
    out["wieferich_base2"] = [int(m.group(1)), int(m.group(2))]
    r = src("A007508/README.md")
    m = re.search(r"a\(n\) = #.*?\n\n(.*?)\n\n", r, re.S)
    out["twins_below_10n"] = [int(x) for x in re.findall(r"\d+", m.group(1))]
    g = src("A158939/a158939.c")
    m = re.search(r"Known terms \(offset 1, n = 1\.\.17\):\n(.*?)\n \* a\(16\)", g, re.S)
    out["A158939"] = [int(x) for x in re.findall(r"\d+", m.group(1))]
    g = src("A252768/a252768.c")
    m = re.search(r"Terms: a\(1\.\.7\) = ([\d, ]+) \(OEIS, 2014\);\n \*\s+a\(8\) = (\d+) and a\(9\) = (\d+)", g)
    out["A252768"] = [int(x) for x in m.group(1).split(",")] + [int(m.group(2)), int(m.group(3))]
    g = src("gapchain/README.md")
    sec = g.split("## Relation to OEIS A016045", 1)[1].split("\n## ", 1)[0]
    rows = re.findall(r"^\|\s*(\d+)\s*\|\s*(\d+)\s*\|\s*\**([\d,]+)\**", sec, re.M)
    out["A016045"] = [int(v.replace(",", "")) for n, l, v in rows]
    sec = g.split("## Decreasing gaps: OEIS A263049", 1)[1].split("\n## ", 1)[0]
    rows = re.findall(r"^\|\s*(\d+)\s*\|\s*(\d+)\s*\|\s*\**([\d,]+)\**", sec, re.M)
    out["A263049"] = [int(v.replace(",", "")) for n, l, v in rows]
    return out


def run_py(script, *args):
    r = subprocess.run([sys.executable, os.path.join(REF, script), *map(str, args)], capture_output=True, text=True,
                       check=True)
    return r.stdout.strip()


def verify_py():
    out = {"wieferich_base2": [], "sext": []}
    for lo, hi in [(10 ** 12, 10 ** 12 + 100000), (10 ** 15, 10 ** 15 + 50000), (2 ** 62 - 40000, 2 ** 62),
                   (1000, 200000), (0, 5000)]:
        line = run_py("A001220/verify_wieferich.py", "range", lo, hi, 2)
        _, a, b, cnt, kv = line.split()
        out["wieferich_base2"].append({"lo": int(a), "hi": int(b), "primes": int(cnt), "cks": int(kv.split(":")[1], 16)})
    for lo, hi in [("1e15", "1e15+2e10"), ("1e9", "1e9+4e9"), ("0", "1e8")]:
        line = run_py("A350826/verify_a350826.py", "count", lo, hi)
        m = re.search(r"(\d+)\s+cks\s+([0-9a-f]+)", line)
        out["sext"].append({"lo": lo, "hi": hi, "count": int(m.group(1)), "cks": int(m.group(2), 16)})
    return out


def stats_hash(blocks):
    arr = np.stack([blocks[n] for n in blocks.dtype.names], axis=1)
    return fnv_u64s(arr.reshape(-1))


def configs():
    t = oracle.threads()
    out = {}
    # config 1
    t0 = time.time()
    lo, hi = 10 ** 9, 10 ** 9 + 10 ** 8
    r = oracle.sieve_range(lo, hi, hash_log2=19, nthreads=t)
    out["config1"] = {"lo": lo, "hi": hi, "hash_log2": 19,
                      "stats": {k: r[k] for k in oracle.STATS_FIELDS},
                      "hashes": [int(x) for x in r["hashes"]]}
    print("config1", time.time() - t0, flush=True)
    # config 2
    t0 = time.time()
    lo, hi = 10 ** 15, 10 ** 15 + 2 ** 34
    r = oracle.sieve_range(lo, hi, block_log2=24, hash_log2=20, nthreads=t)
    blocks = r["blocks"]
    samp = [0, 1, 511, 512, 1023]
    out["config2"] = {"lo": lo, "hi": hi, "block_log2": 24, "hash_log2": 20,
                      "stats": {k: r[k] for k in oracle.STATS_FIELDS},
                      "nblocks": len(blocks), "blocks_fnv": stats_hash(blocks),
                      "blocks_sample": {str(i): {n: int(blocks[i][n]) for n in blocks.dtype.names} for i in samp},
                      "nhashes": len(r["hashes"]), "hashes_fnv": fnv_u64s(r["hashes"]),
                      "hashes_sample": {str(i): int(r["hashes"][i]) for i in [0, 1, 8191, 16383]}}
    c, k = oracle.ref_count_sext(lo, hi, t)
    if (c, k) != (r["tuple6"], r["tuple6_cks"]):
        raise SystemExit(f"config2 6-tuples: oracle {r['tuple6']} {r['tuple6_cks']:x} vs reference {c} {k:x}")
    out["config2"]["reference_tuple6"] = {"count": c, "cks": k}
    print("config2", time.time() - t0, flush=True)
    # config 3
    t0 = time.time()
    sys.path.insert(0, ROOT)
    import mathpub_b200 as mp
    n, lens = mp.bpsw_workload(0x3C0FFEE, 1 << 26, 4096)
    v = oracle.bpsw(n, t)
    vr = oracle.ref_bpsw(n, t)
    if not np.array_equal(v, vr):
        raise SystemExit("config3: oracle and reference verdicts differ")
    packed = np.packbits(v, bitorder="little")
    offs = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    per_list = np.add.reduceat(v.astype(np.int64), offs[:-1]) if len(lens) else np.zeros(0)
    out["config3"] = {"seed": 0x3C0FFEE, "count": 1 << 26, "nlists": 4096,
                      "inputs_fnv": fnv_u64s(n), "lens_fnv": fnv_u64s(lens.astype(np.uint64)),
                      "primes": int(v.sum()), "verdict_fnv": fnv_bytes(packed.tobytes()),
                      "per_list_primes_fnv": fnv_u64s(per_list.astype(np.uint64)),
                      "lens_head": [int(x) for x in lens[:8]]}
    print("config3", time.time() - t0, flush=True)
    # config 4
    t0 = time.time()
    lo, hi = 10 ** 12, 10 ** 12 + 4 * 10 ** 9
    w = oracle.wieferich_range(lo, hi, t)
    p, k, f = oracle.ref_wieferich_scan(lo, hi, t)
    if (p, k, f) != (w["primes"], w["cks"], 0):
        raise SystemExit(f"config4: oracle {w['primes']} {w['cks']:x} vs reference {p} {k:x} flt {f}")
    out["config4"] = {"lo": lo, "hi": hi, **w, "reference": {"primes": p, "cks": k}}
    print("config4", time.time() - t0, flush=True)
    return out


def main():
    oracle.build(ref=True)
    rv = ref_vectors()
    with open(os.path.join(HERE, "ref_vectors.json"), "w") as f:
        json.dump(rv, f, indent=1)
    print("ref_vectors ok", flush=True)
    vp = verify_py()
    with open(os.path.join(HERE, "verify_py.json"), "w") as f:
        json.dump(vp, f, indent=1)
    print("verify_py ok", flush=True)
    if "--skip-full" not in sys.argv:
        cf = configs()
        with open(os.path.join(HERE, "configs.json"), "w") as f:
            json.dump(cf, f, indent=1)
    print("done")


if __name__ == "__main__":
    main()
