"""Chunk logs in the reference tools' formats (mathpub_b200/chunklog.py), compared with the logs
that the reference tools write themselves: A001220/wieferich.c -L (base 2) and
A007508/a007508.c -l, both built from the reference sources against the CPU stand-in for
primesieve (oracle/_ref).  On the CPU the log writers run on an oracle-backed engine (host
logic); on the GPU on the real one.  The last test runs A007508 compiled unmodified against
the primesieve drop-in, whose ps and iter kernels then count on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
W_LO, W_HI, W_CHUNK = 10 ** 12, 10 ** 12 + 2 * 10 ** 8, 5 * 10 ** 7
T_N, T_CHUNK = 9, 3 * 10 ** 7


def tool(name):
    p = os.path.join(REF_BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} is not built (oracle/_ref)")
    return p


def reference_wieferich_log(tmp_path):
    log = tmp_path / "w.log"
    subprocess.run([tool("wieferich_cpu"), "scan", str(W_LO), str(W_HI), "-b", "2", "-c", str(W_CHUNK), "-L", str(log),
                    "-q", "-t", "8"], check=True, capture_output=True, timeout=600)
    return log.read_text().splitlines()


def reference_twin_log(tmp_path):
    log = tmp_path / "t.log"
    subprocess.run([tool("a007508_cpu"), str(T_N), "-s", str(T_CHUNK), "-l", str(log), "-t", "8"], check=True,
                   capture_output=True, timeout=600)
    return log.read_text().splitlines()


def same_log(ours, theirs):
    # the tool appends chunk lines in completion order (threads); the decade lines in order
    assert sorted(l for l in ours if l.startswith("k")) == sorted(l for l in theirs if l.startswith("k"))
    assert [l for l in ours if l.startswith("d")] == [l for l in theirs if l.startswith("d")]


class OracleEngine:
    """The two engine calls the log writers make, answered by the oracle (CPU)."""

    def __init__(self, orc):
        self.o = orc

    def wieferich_range(self, lo, hi):
        return self.o.wieferich_range(lo, hi)

    def sieve_range(self, lo, hi):
        return self.o.sieve_range(lo, hi)


def test_chunk_geometry_matches_a007508():
    from mathpub_b200 import chunklog
    assert [chunklog.kbound(n) for n in range(4)] == [0, 0, 3, 33]
    assert chunklog.default_chunk_k(9) == 10 ** 9 // 30 and chunklog.default_chunk_k(19) == 10 ** 13 // 30


def test_wieferich_log_host_logic(orc, tmp_path):
    from mathpub_b200 import chunklog
    ours = list(chunklog.wieferich_lines(OracleEngine(orc), W_LO, W_HI, W_CHUNK))
    assert ours == reference_wieferich_log(tmp_path)


def test_twin_log_host_logic(orc, tmp_path):
    from mathpub_b200 import chunklog
    same_log(list(chunklog.twin_lines(OracleEngine(orc), T_N, T_CHUNK)), reference_twin_log(tmp_path))


@pytest.mark.gpu
def test_wieferich_log_on_gpu(engine, tmp_path):
    from mathpub_b200 import chunklog
    assert list(chunklog.wieferich_lines(engine, W_LO, W_HI, W_CHUNK)) == reference_wieferich_log(tmp_path)


@pytest.mark.gpu
def test_twin_log_on_gpu(engine, tmp_path):
    from mathpub_b200 import chunklog
    same_log(list(chunklog.twin_lines(engine, T_N, T_CHUNK)), reference_twin_log(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["ps", "iter"])
def test_a007508_on_the_dropin(kernel):
    """a(1..10) from A007508 compiled against the drop-in (count_twins or iterators on the GPU)
    and from its own twin kernel on the CPU."""
    def terms(out):
        return [tuple(l.split()[:2]) for l in out.splitlines() if l and not l.startswith("#")]
    gpu = subprocess.run([tool("a007508_gpu"), "10", "-k", kernel, "-t", "4"], capture_output=True, text=True,
                         timeout=600)
    cpu = subprocess.run([tool("a007508_cpu"), "10", "-t", "8"], capture_output=True, text=True, timeout=600)
    assert gpu.returncode == 0 and cpu.returncode == 0, (gpu.stderr[-500:], cpu.stderr[-500:])
    assert terms(gpu.stdout) == terms(cpu.stdout)
    assert terms(cpu.stdout)[-1] == ("10", "27412679")                  # A007508(10), A007508/README.md
