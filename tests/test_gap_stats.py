"""Statistics of the prime-gap stream (mp_gap_stats_range): the gap histogram (A252768's power
sums) and the run lengths of A158939.

CPU: the oracle's restatement is pinned to the reference's published terms (A158939
a(1..10), A252768 a(1..5)) and to the run-length table that the reference's own
A158939/a158939.c prints for [0, 10^9) (built from its source against the CPU stand-in).
GPU: the engine agrees with the oracle on several ranges, finds A158939 a(1..13) by
scanning [0, 10^12), reproduces the reference tool's table for [0, 10^9), and the reference
tool compiled unmodified against the primesieve drop-in prints the same results as on the CPU."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def tool(name):
    p = os.path.join(REF_BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} is not built (oracle/_ref)")
    return p


def a158939_scan(exe, end):
    r = subprocess.run([exe, "scan", "0", str(end), "-t", "8", "-q", "-c", "100000000"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    return r.stdout


def parse_table(out):
    """{n: primes with L(p) = n} from the tool's run-length distribution table."""
    tab = {}
    body = out.split("run-length distribution", 1)[1]
    for m in re.finditer(r"^\s+(\d+)\s+(\d+)\s+\S+\s+\S+\s*$", body, re.M):
        tab[int(m.group(1))] = int(m.group(2))
    return tab


def timing_free(out):
    return [l for l in out.splitlines() if "numbers/s" not in l and not l.startswith("#")]


def power_sums(gap_hist, kmax):
    g = np.arange(len(gap_hist), dtype=object) * 2
    g[0] = 1                                                  # bin 0: the gap 1 of p = 2
    c = [int(x) for x in gap_hist]
    return [sum(ci * int(gi) ** k for ci, gi in zip(c, g) if ci) for k in range(1, kmax + 1)]


# ---- CPU: the oracle pinned ----

def test_oracle_finds_a158939_terms(orc, ref_vectors):
    g = orc.gap_stats(0, 10 ** 8)
    assert [int(x) for x in g["run_first"][1:11]] == ref_vectors["A158939"][:10]
    assert g["unsettled"] == 0


def test_oracle_matches_reference_run_table(orc):
    tab = parse_table(a158939_scan(tool("a158939_cpu"), 10 ** 8))
    g = orc.gap_stats(0, 10 ** 8)
    assert {n: int(g["run_hist"][n]) for n in tab} == tab


def test_oracle_gaps_give_a252768_terms(orc, ref_vectors):
    """A252768: the smallest prime p whose power sums S_k(p) = sum of g^k over the gaps
    between the primes <= p are prime for k = 1..n (A252768/a252768.c:11-22)."""
    p = orc.primes_range(0, 400000).astype(np.uint64)
    g = np.diff(p)
    depth = np.zeros(len(p), dtype=np.int64)
    alive = np.ones(len(p), dtype=bool)
    alive[0] = False                                          # p = 2: no gap below it
    for k in range(1, 6):
        s = np.concatenate([[0], np.cumsum(g.astype(np.uint64) ** np.uint64(k))])   # S_k(p_i)
        prime = np.zeros(len(p), dtype=bool)
        nz = s >= 2
        prime[nz] = orc.bpsw(s[nz].astype(np.uint64))
        alive &= prime
        depth[alive] = k
    a = [int(p[np.argmax(depth >= n)]) for n in range(1, 6)]
    assert a == ref_vectors["A252768"][:5]


# ---- GPU ----

@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi", [(0, 10 ** 7), (10 ** 9, 10 ** 9 + 10 ** 8), (10 ** 15, 10 ** 15 + 5 * 10 ** 7),
                                   (2 ** 50 - 10 ** 6, 2 ** 50 + 10 ** 7), (1, 2), (2, 3), (3, 1000)])
def test_gap_stats_match_oracle(engine, orc, lo, hi):
    got, want = engine.gap_stats(lo, hi), orc.gap_stats(lo, hi)
    assert np.array_equal(got["gap_hist"], want["gap_hist"])
    assert np.array_equal(got["run_hist"], want["run_hist"])
    assert np.array_equal(got["run_first"], want["run_first"])
    assert got["unsettled"] == want["unsettled"] == 0
    assert power_sums(got["gap_hist"], 6) == power_sums(want["gap_hist"], 6)


@pytest.mark.gpu
def test_gpu_scan_finds_a158939_up_to_a13(engine, ref_vectors):
    g = engine.gap_stats(0, 10 ** 12)
    assert [int(x) for x in g["run_first"][1:14]] == ref_vectors["A158939"][:13]
    assert int(g["gap_hist"].sum()) == 37607912018          # pi(10^12), A158939/cuda/a158939_cuda.cu PI10


@pytest.mark.gpu
def test_gpu_matches_reference_run_table():
    tab = parse_table(a158939_scan(tool("a158939_cpu"), 10 ** 9))
    import mathpub_b200 as mp
    e = mp.Engine(0)
    try:
        g = e.gap_stats(0, 10 ** 9)
    finally:
        e.close()
    assert {n: int(g["run_hist"][n]) for n in tab} == tab


@pytest.mark.gpu
def test_reference_a158939_on_the_dropin():
    gpu = a158939_scan(tool("a158939_gpu"), 10 ** 9)
    cpu = a158939_scan(tool("a158939_cpu"), 10 ** 9)
    assert timing_free(gpu) == timing_free(cpu)
