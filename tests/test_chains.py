"""Chains of consecutive primes with gaps 2, 4, 6, ... (A016045; mp_gap_chains and the
chain_hist of mp_gap_stats_range).

CPU: the oracle's chains equal the output of the reference's own gapchain/gapchain_ps.c
(built from its source against the CPU stand-in for primesieve), and give the first terms of
A016045 from the reference's table.  GPU: the engine agrees with the oracle, finds A016045
a(1..11) by scanning [0, 4.7e12), and gapchain_ps compiled unmodified against the primesieve
drop-in (both directions, so prev_prime too) prints the same chains as on the CPU."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
EXTRA = 8                                        # gapchain_ps reports lengths k .. k + 8 (the last with " +")


def tool(name):
    p = os.path.join(REF_BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} is not built (oracle/_ref)")
    return p


def gapchain(exe, k, start, end, gaps="inc"):
    r = subprocess.run([exe, "-l", str(k), "-s", str(start), "-e", str(end), "-t", "8", "-q", "-g", gaps],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    return r.stdout


def inc_chains(out):
    """{head: length} from the tool's increasing-chain lines ("L: p q ..." or "inc L: p ...")."""
    got = {}
    for line in out.splitlines():
        m = re.match(r"^(?:inc )?\s*(\d+): (\d+)", line)
        if m:
            got[int(m.group(2))] = int(m.group(1))
    return got


def capped(heads, lens, k):
    return {int(h): min(int(l), k + EXTRA) for h, l in zip(heads, lens)}


def first_heads(heads, lens, lengths):
    return [int(heads[np.argmax(lens >= L)]) if (lens >= L).any() else 0 for L in lengths]


# ---- CPU ----

def test_oracle_matches_gapchain_ps(orc):
    out = gapchain(tool("gapchain_ps_cpu"), 5, 3, 10 ** 8)
    heads, lens = orc.gap_chains(3, 10 ** 8 + 1, 5)
    assert capped(heads, lens, 5) == inc_chains(out)
    assert len(heads) == 1538


def test_oracle_first_chains_are_a016045(orc, ref_vectors):
    heads, lens = orc.gap_chains(0, 2 * 10 ** 8, 2)
    assert first_heads(heads, lens, range(2, 10)) == ref_vectors["A016045"][:8]


# ---- GPU ----

@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi,k", [(0, 10 ** 6, 2), (3, 10 ** 8 + 1, 5), (10 ** 12, 10 ** 12 + 10 ** 9, 4),
                                     (2 ** 60 - 10 ** 9, 2 ** 60, 4)])
def test_chains_match_oracle(engine, orc, lo, hi, k):
    gh, gl = engine.gap_chains(lo, hi, k)
    oh, ol = orc.gap_chains(lo, hi, k)
    assert np.array_equal(gh, oh) and np.array_equal(gl, ol)
    assert np.array_equal(engine.gap_stats(lo, hi)["chain_hist"], orc.gap_stats(lo, hi)["chain_hist"])


@pytest.mark.gpu
def test_gpu_finds_a016045_up_to_a11(engine, ref_vectors):
    small = engine.gap_chains(0, 10 ** 5, 2)
    big = engine.gap_chains(0, 47 * 10 ** 11, 7)
    firsts = first_heads(*small, range(2, 7)) + first_heads(*big, range(7, 13))
    assert firsts == ref_vectors["A016045"][:11]


@pytest.mark.gpu
def test_reference_gapchain_ps_on_the_dropin():
    gpu = gapchain(tool("gapchain_ps_gpu"), 5, 3, 10 ** 9, "both")
    cpu = gapchain(tool("gapchain_ps_cpu"), 5, 3, 10 ** 9, "both")
    assert sorted(gpu.splitlines()) == sorted(cpu.splitlines())
    assert sum(1 for l in cpu.splitlines() if l.startswith("dec")) > 100
