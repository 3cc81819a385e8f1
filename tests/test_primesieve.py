"""The primesieve drop-in (include/primesieve.h on libmathpub.so).

On the CPU: the library exports every function the header declares, a C program compiled
against the header links, and without a GPU every call reports an error (no CPU fallback).
On the GPU: the iterator (next_prime / prev_prime / generate_next_primes, across many buffer
refills and in both directions), generate_primes, generate_n_primes, count_primes and
count_twins agree with the oracle; and the reference's own A000230/a000230.c, compiled
unmodified against the drop-in, prints the same terms as when it is compiled against the CPU
stand-in for primesieve."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "primesieve.h")
LIBDIR = os.path.join(ROOT, "mathpub_b200")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
MASK = (1 << 64) - 1


def declared():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    src = re.sub(r"static inline[^{]*\{.*?\n\}", "", src, flags=re.S)      # header-only helpers
    return sorted(set(re.findall(r"\b(primesieve_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    from mathpub_b200 import build
    build.build()
    exe = str(tmp_path_factory.mktemp("ps") / "primesieve_harness")
    subprocess.run(["gcc", "-O2", "-std=gnu11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "primesieve_harness.c"), "-o", exe, "-L", LIBDIR, "-lmathpub",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def run(exe, *args):
    out = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


def summary(p):
    """n, first, last, sum of p, sum of i * p (mod 2^64) of a sequence, as the harness prints."""
    p = np.asarray(p, dtype=np.uint64)
    n = len(p)
    if not n:
        return {"n": 0, "first": 0, "last": 0, "s1": 0, "s2": 0}
    s1 = int(p.sum(dtype=np.uint64))
    s2 = int((p * np.arange(n, dtype=np.uint64)).sum(dtype=np.uint64))
    return {"n": n, "first": int(p[0]), "last": int(p[-1]), "s1": s1 & MASK, "s2": s2 & MASK}


def check(got, want):
    assert got["err"] == 0, got
    for k in ("n", "first", "last", "s1", "s2"):
        assert got[k] == want[k], (k, got, want)


# ---- CPU ----

def test_header_functions_are_exported():
    from mathpub_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (primesieve_[a-z0-9_]+)\b", out))
    names = declared()
    assert "primesieve_generate_next_primes" in names and "primesieve_next_prime" not in names
    missing = [f for f in names if f not in exported]
    assert not missing, missing


def test_without_gpu_every_call_reports_an_error(harness):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    r = run(harness, "next", 0, 100, 10)
    assert r["err"] == 1 and r["last"] == MASK
    assert run(harness, "count", 0, 1000)["err"] == 1
    assert run(harness, "gen", 0, 1000, 64)["err"] == 1


# ---- GPU ----

@pytest.mark.gpu
@pytest.mark.parametrize("start,hint,count", [
    (0, 1000, 400000),                       # from 2 on, through eight refills of growing size
    (10 ** 12 + 12345, 10 ** 12 + 10 ** 6, 300000),
    (2 ** 50 - 10 ** 6, 2 ** 50, 200000),
    (7, 6, 5000),                            # a hint below start
])
def test_next_prime_walk(harness, orc, start, hint, count):
    got = run(harness, "next", start, hint, count)
    span = 64
    while True:
        p = orc.primes_range(start, start + span * count)
        if len(p) >= count:
            break
        span *= 2
    check(got, summary(p[:count]))


@pytest.mark.gpu
@pytest.mark.parametrize("start,count", [(10 ** 9 + 7, 200000), (100, 1000), (2 ** 40 + 1, 100000)])
def test_prev_prime_walk(harness, orc, start, count):
    got = run(harness, "prev", start, count)
    lo = max(0, start - 64 * count)
    p = orc.primes_range(lo, start + 1)[::-1]
    want = list(p[:count])
    if len(want) < count:
        want.append(0)                       # primesieve's "no prime below"
    check(got, summary(want))


@pytest.mark.gpu
def test_generate_next_primes_buffer(harness, orc):
    lo, hi = 10 ** 10, 10 ** 10 + 3 * 10 ** 7
    check(run(harness, "buffer", lo, hi), summary(orc.primes_range(lo, hi)))


@pytest.mark.gpu
def test_mixed_directions(harness, orc):
    start = 10 ** 15 + 1
    around = orc.primes_range(start - 10 ** 4, start + 10 ** 4)
    i = int(np.searchsorted(around, start))            # first prime >= start
    seq = [around[i], around[i + 1], around[i + 2]]     # next x3
    k = i + 2
    for _ in range(5):                                  # prev x5
        k -= 1
        seq.append(around[k])
    for _ in range(10):                                 # next x10
        k += 1
        seq.append(around[k])
    check(run(harness, "mixed", start), summary(seq))


@pytest.mark.gpu
def test_generate_primes_and_n_primes(harness, orc):
    lo, hi = 10 ** 9, 10 ** 9 + 10 ** 7
    want = summary(orc.primes_range(lo, hi + 1))
    check(run(harness, "gen", lo, hi, 64), want)
    check(run(harness, "gen", lo, hi, 32), want)
    p = orc.primes_range(10 ** 14, 10 ** 14 + 5 * 10 ** 6)
    check(run(harness, "genn", 100000, 10 ** 14), summary(p[:100000]))


@pytest.mark.gpu
@pytest.mark.parametrize("a,b", [(0, 10 ** 9), (10 ** 15, 10 ** 15 + 2 * 10 ** 8), (3, 5), (4, 6)])
def test_count_primes_and_twins(harness, orc, ref_vectors, a, b):
    r = run(harness, "count", a, b)
    assert r["err"] == 0
    assert r["n"] == orc.sieve_range(a, b + 1)["pi"]
    # twin pairs with both members in [a, b]: first members in [a, b - 1)
    assert r["s1"] == (orc.sieve_range(a, b - 1)["twins"] if b - 1 > a else 0)
    if (a, b) == (0, 10 ** 9):
        assert r["n"] == 50847534                            # pi(1e9), A001220/wieferich.c:1851


@pytest.mark.gpu
def test_past_the_max_stop_is_an_error(harness):
    r = run(harness, "top")
    assert r["first"] == 2 ** 64 - 2 ** 18 - 1
    assert r["err"] == 1 and r["last"] == MASK


@pytest.mark.gpu
def test_reference_a000230_links_unmodified():
    """A000230 (smallest prime starting a gap of 2n), the reference's own program with its
    worker threads and primesieve iterators, on the GPU drop-in and on the CPU stand-in."""
    gpu, cpu = os.path.join(REF_BIN, "a000230_gpu"), os.path.join(REF_BIN, "a000230_cpu")
    if not (os.path.exists(gpu) and os.path.exists(cpu)):
        pytest.skip("the reference builds in oracle/_ref are absent")
    a = subprocess.run([gpu, "-n", "150", "-t", "8"], capture_output=True, text=True, timeout=600)
    b = subprocess.run([cpu, "-n", "150", "-t", "8"], capture_output=True, text=True, timeout=600)
    assert a.returncode == 0 and b.returncode == 0, (a.stderr[-500:], b.stderr[-500:])
    assert a.stdout == b.stdout
    assert len(a.stdout.splitlines()) == 150
