"""The reference's GPU constellation search on this library: gapchain/gapsieve_cuda_host.c
(with gapchain/gapsieve.c) compiled unmodified and linked against libmathpub's cu_* entry points
(include/gapsieve_cuda.h) in place of the reference's gapsieve_cuda.cu.

CPU: the library exports every entry point of the interface.
GPU: cu_sprp_batch agrees with a base-2 strong test in Python's integers, below and above
2^64; and the reference program on the GPU alone (-t 0 --gpu) prints exactly the chains, and
the same counts by length, as the reference's CPU build, for both shapes, from 3 up, around
the A016045 a(15) record, across 2^64 and at 1e20."""
import os
import random
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
ENTRY = ["cu_init", "cu_tables", "cu_shape", "cu_slot", "cu_grow", "cu_submit", "cu_wait", "cu_list",
         "cu_sprp_batch"]


def test_library_exports_the_gapsieve_interface():
    src = open(os.path.join(ROOT, "include", "gapsieve_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    assert sorted(set(re.findall(r"\b(cu_[a-z0-9_]+)\s*\(", src))) == sorted(ENTRY)
    from mathpub_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (cu_[a-z0-9_]+)\b", out))
    assert set(ENTRY) <= exported


def test_interface_refuses_to_run_without_a_gpu():
    """No CPU fallback: without a GPU, cu_init fails, and the reference's host then reports that
    it cannot use the GPU (gapchain/gapsieve_cuda_host.c:91-92)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    import ctypes as C
    import mathpub_b200 as mp
    L = mp.lib()
    L.cu_init.argtypes = [C.c_char_p, C.c_size_t]
    name = C.create_string_buffer(64)
    assert L.cu_init(name, 64) != 0


def sprp2(n):
    if n == 2:
        return True
    if n < 3 or n % 2 == 0:
        return False
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    x = pow(2, d, n)
    if x in (1, n - 1):
        return True
    for _ in range(s - 1):
        x = x * x % n
        if x == n - 1:
            return True
    return False


@pytest.mark.gpu
def test_sprp_batch_matches_python():
    import ctypes as C
    import mathpub_b200 as mp
    L = mp.lib()
    L.cu_init.argtypes = [C.c_char_p, C.c_size_t]
    L.cu_sprp_batch.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
    name = C.create_string_buffer(128)
    assert L.cu_init(name, 128) == 0 and b"B200" in name.value
    rng = random.Random(2024)
    ns = [0, 1, 2, 3, 4, 9, 2047, 3215031751, 3825123056546413051, 2 ** 64 - 59, 2 ** 64 + 13, 2 ** 89 - 1,
          2 ** 127 - 1, 2 ** 61 - 1, (1 << 64) + 1, 1797761 * 3595521, 4294967291 * 8589934583 * 4294967279]
    for bits in (20, 40, 63, 64, 65, 70, 82, 96, 110, 126):
        ns += [rng.getrandbits(bits) | 1 for _ in range(400)]
    arr = np.zeros((len(ns), 2), dtype=np.uint64)
    for i, n in enumerate(ns):
        assert n < 2 ** 127
        arr[i, 0], arr[i, 1] = n & (2 ** 64 - 1), n >> 64
    ok = np.zeros(len(ns), dtype=np.uint8)
    assert L.cu_sprp_batch(arr.ctypes.data, len(ns), ok.ctypes.data) == 0
    assert [bool(x) for x in ok] == [sprp2(n) for n in ns]


def run(exe, args, log=None, env=None):
    p = os.path.join(REF, exe)
    if not os.path.exists(p):
        pytest.skip(f"oracle/_ref/{exe} is not built")
    extra = ["--log", str(log)] if log else []
    r = subprocess.run([p, *args.split(), "-q", *extra], capture_output=True, text=True, timeout=900,
                       env={**os.environ, **(env or {})})
    assert r.returncode == 0, r.stderr[-600:]
    # the host redoes a failed GPU unit and then searches it on the CPU (exactly), which would
    # hide a GPU failure from the comparison; the GPU must have done every unit
    assert "on the CPU" not in r.stderr
    if log:
        assert "failed" not in open(log).read()
    # the summary: counts by length, or the --first answer; without the header line (it names
    # the CPU threads or the GPU), the progress line and durations
    summary = [re.sub(r"\d+:\d\d:\d\d", "", line) for line in r.stderr.splitlines()
               if not line.startswith("consecutive primes") and "elapsed" not in line]
    return sorted(r.stdout.splitlines()), summary


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    "-l 16 -s 1397388433200922807 -e 1397408433200922807",
    "-l 9 -g both -s 1000000000000000 -e 1000100000000000",
    "-l 5 -g both -s 3 -e 30000000000",
    "-l 10 -g both -s 18446739073709551616 -e 18446749073709551616",     # 2^64 -+ 5e12
    "-l 10 -g both -s 100000000000000000000 -e 100000010000000000000",
    "-l 15 -s 221860000000000000 -e 221870000000000000 --first",
])
def test_reference_gapsieve_on_the_gpu_matches_its_cpu_build(args, tmp_path):
    cpu_lines, cpu_counts = run("gapsieve_cpu", args)
    gpu_lines, gpu_counts = run("gapsieve_gpu", args + " -t 0 --gpu", log=tmp_path / "gpu.log")
    assert len(cpu_lines) > 0
    assert gpu_lines == cpu_lines
    assert gpu_counts == cpu_counts


@pytest.mark.gpu
@pytest.mark.parametrize("env", [{"GAPSIEVE_GPU_CAP": "1000"}, {"GAPSIEVE_GPU_SPLIT": "0", "GAPSIEVE_GPU_UNIT": "3"}])
def test_reference_host_protocol_paths(env, tmp_path):
    """The host's own switches (gapchain/gapsieve_cuda_host.c:18-21): lists of 1000 entries
    overflow on every unit, so the host enlarges them with cu_grow and resubmits; SPLIT 0 sends
    every member to the tail kernel, in units of three segments."""
    args = "-l 9 -g both -s 1000000000000000 -e 1000100000000000"
    cpu_lines, cpu_counts = run("gapsieve_cpu", args)
    gpu_lines, gpu_counts = run("gapsieve_gpu", args + " -t 0 --gpu", log=tmp_path / "gpu.log", env=env)
    assert (gpu_lines, gpu_counts) == (cpu_lines, cpu_counts)
    if "GAPSIEVE_GPU_CAP" in env:
        assert "enlarged" in open(tmp_path / "gpu.log").read()
