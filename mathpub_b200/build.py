"""Build recipe for libmathpub.so (all CUDA sources, sm_100a) next to this file.

    python -m mathpub_b200.build          # or: from mathpub_b200.build import build; build()

nvcc compiles for the B200 only (-gencode arch=compute_100a,code=sm_100a) with -lineinfo;
the library is rebuilt when a source or header is newer than it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmathpub.so")
WORK = os.path.join(HERE, "libmpwork.so")
SOURCES = ["mp_api.cu", "mp_sieve.cu", "mp_bpsw.cu", "mp_fermat.cu", "mp_tune.cu", "mp_serve.cu", "mp_probe.cu",
           "mp_primesieve.cu", "mp_gap.cu", "mp_chain.cu"]
HEADERS = ["mp_common.cuh", "mp_mont64.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", h)
                                                                  for h in ("mathpub_gpu.h", "primesieve.h", "gapsieve_cuda.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build_work(force=False):
    """libmpwork.so: the seeded workload generators (plain C)."""
    src = os.path.join(CSRC, "mp_workload.c")
    if not force and os.path.exists(WORK) and os.path.getmtime(WORK) >= os.path.getmtime(src):
        return WORK
    cc = os.environ.get("CC", "gcc")
    r = subprocess.run([cc, "-O2", "-std=gnu11", "-fPIC", "-shared", "-o", WORK + ".tmp", src],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("building libmpwork.so failed")
    os.replace(WORK + ".tmp", WORK)
    return WORK


def build(force=False, verbose=False, extra=()):
    build_work(force)
    if not force and not _stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [NVCC, *FLAGS, *extra, "-shared", "-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libmathpub.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=("-Xptxas", "-v") if "--ptxas-v" in sys.argv else ())
    print(LIB)
