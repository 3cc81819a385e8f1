"""Checkpoint files in the reference tools' formats (mathpub_b200/checkpoint.py), checked against
the reference's own A001220/wieferich.c built from its source against the CPU stand-in for
primesieve (oracle/_ref/wieferich_cpu): the state written here after every chunk equals the
state the tool writes at the end of its own scan, and the tool resumed from a state written
here after part of the chunks ends with the summary and state of a scan that ran alone.  On
the CPU the writer runs on an oracle-backed engine (host logic); on the GPU on the real one."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
LO, HI, CHUNK = 10 ** 12, 10 ** 12 + 2 * 10 ** 8, 5 * 10 ** 7          # four chunks


def tool():
    p = os.path.join(REF_BIN, "wieferich_cpu")
    if not os.path.exists(p):
        pytest.skip("wieferich_cpu is not built (oracle/_ref)")
    return p


def scan(state, hi=HI):
    """The reference tool's base-2 scan with the checkpoint file `state`; its stdout."""
    r = subprocess.run([tool(), "scan", str(LO), str(hi), "-b", "2", "-c", str(CHUNK), "-S", str(state), "-q", "-t",
                        "8"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    return r.stdout


def summary(out):
    return [l for l in out.splitlines() if l.startswith(("SUMMARY", "base"))]


class OracleEngine:
    def __init__(self, orc):
        self.o = orc

    def wieferich_range(self, lo, hi):
        return self.o.wieferich_range(lo, hi)


def check(engine, tmp_path):
    from mathpub_b200 import checkpoint
    alone = tmp_path / "alone.state"
    out_alone = scan(alone)
    # the state after every chunk is the one the tool writes at the end of its own scan
    assert checkpoint.wieferich_state(engine, LO, HI, CHUNK, 4) == alone.read_text()
    # the tool resumes from a state written here after two of the four chunks
    part = tmp_path / "part.state"
    checkpoint.write_atomically(str(part), checkpoint.wieferich_state(engine, LO, HI, CHUNK, 2))
    out_resumed = scan(part)
    assert summary(out_resumed) == summary(out_alone)
    assert part.read_text() == alone.read_text()
    # and the other way round: the tool's state after two chunks is the one written here
    half = tmp_path / "half.state"
    scan(half, hi=LO + 2 * CHUNK)
    text = half.read_text().replace(f"end {LO + 2 * CHUNK}\n", f"end {HI}\n")
    assert text == checkpoint.wieferich_state(engine, LO, HI, CHUNK, 2)


def test_wieferich_state_host_logic(orc, tmp_path):
    check(OracleEngine(orc), tmp_path)


def test_wieferich_state_rejects_bad_frontier(orc):
    from mathpub_b200 import checkpoint
    with pytest.raises(ValueError):
        checkpoint.wieferich_state(OracleEngine(orc), LO, HI, CHUNK, 5)


@pytest.mark.gpu
def test_wieferich_state_on_gpu(engine, tmp_path):
    check(engine, tmp_path)
