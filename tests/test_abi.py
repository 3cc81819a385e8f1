"""The C ABI boundary on the CPU: libmathpub.so loads and exports every entry point that
include/mathpub_gpu.h declares, refuses to run without a GPU (no CPU fallback), and the
seeded workload generator is deterministic.  No compute call needs a GPU here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mathpub_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mp_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    f = declared_functions()
    for name in ["mp_init", "mp_free", "mp_last_error", "mp_sieve_range", "mp_bpsw_u64", "mp_bpsw_batches",
                 "mp_fermat_q_base2", "mp_wieferich_range", "mp_serve_open", "mp_serve_submit_range",
                 "mp_serve_submit_bpsw", "mp_serve_poll", "mp_serve_close", "mp_autotune"]:
        assert name in f


def test_library_builds_and_exports_every_symbol():
    from mathpub_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mp_[a-z0-9_]+)\b", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    # the build compiles for sm_100a only: one -gencode, for the B200
    gencodes = [build.FLAGS[i + 1] for i, f in enumerate(build.FLAGS) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]


def test_python_constants_match_the_header():
    import mathpub_b200 as mp
    src = open(os.path.join(ROOT, "include", "mathpub_gpu.h")).read()
    m = re.search(r"#define MP_NOALLOC_MAX_COUNT \(1u << (\d+)\)", src)
    assert m and mp.NOALLOC_MAX_COUNT == 1 << int(m.group(1))


def test_library_loads_and_fails_loudly_without_gpu():
    import mathpub_b200 as mp
    L = mp.lib()
    assert L.mp_version() == 100
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(mp.MathpubError):
        mp.Engine(0)


def test_geometry_helpers():
    import mathpub_b200 as mp
    L = mp.lib()
    lo, hi = 10 ** 9, 10 ** 9 + 10 ** 8
    assert L.mp_sieve_nhashes(lo, hi, 19) == 191
    assert L.mp_sieve_nblocks(10 ** 15, 10 ** 15 + 2 ** 34, 24) == 1024
    assert L.mp_sieve_nwords(lo, hi) == (5 * 10 ** 7 + 63) // 64
    assert L.mp_sieve_nhashes(3, 5, 4) == 1 and L.mp_sieve_nblocks(5, 5, 20) == 0


def test_workload_generator_deterministic(configs):
    import mathpub_b200 as mp
    from helpers import fnv1a64
    n, lens = mp.bpsw_workload(0x3C0FFEE, 1 << 16, 64)
    n2, lens2 = mp.bpsw_workload(0x3C0FFEE, 1 << 16, 64)
    assert np.array_equal(n, n2) and np.array_equal(lens, lens2)
    assert int(lens.sum()) == 1 << 16 and (n & 1).all()
    # the mix (60 / 30 / 10 %): uniform in [2^40, 2^64) and semiprimes near 2^62 are >= 2^40;
    # only the small Chernick numbers (k small) fall below
    frac_big = float(((n >> np.uint64(40)) > 0).mean())
    assert 0.93 < frac_big < 1.0
    c3 = configs["config3"]
    big, blens = mp.bpsw_workload(c3["seed"], c3["count"], c3["nlists"])
    import oracle
    f = int(oracle.o().or_fnv1a64(big.ctypes.data, big.nbytes))
    assert f == c3["inputs_fnv"]
    assert [int(x) for x in blens[:8]] == c3["lens_head"] and int(blens.sum()) == c3["count"]
    assert blens.min() >= 1 and len(blens) == 4096
