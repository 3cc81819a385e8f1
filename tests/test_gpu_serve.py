"""Serving with continuous batching: a mixed stream of range and primality requests gives,
for every request, the same result as the request run alone through the plain entry points."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream(seed, nrange, nbpsw):
    import mathpub_b200 as mp
    rng = np.random.default_rng(seed)
    pool, _ = mp.bpsw_workload(seed, 1 << 16, 0)
    reqs = []
    for _ in range(nrange):
        lo = int(10 ** rng.uniform(9, 18))
        ln = int(2 ** rng.uniform(16, 26))
        reqs.append(("range", lo, lo + ln))
    for _ in range(nbpsw):
        n = int(2 ** rng.uniform(0, 13))
        a = int(rng.integers(0, len(pool) - n))
        reqs.append(("bpsw", pool[a:a + n].copy()))
    order = rng.permutation(len(reqs))
    return [reqs[i] for i in order]


def test_mixed_stream_equals_alone(engine):
    import mathpub_b200 as mp
    reqs = _stream(17, 40, 40)
    with mp.Server(engine, streams=4) as srv:
        ids = []
        for r in reqs:
            ids.append(srv.submit_range(r[1], r[2]) if r[0] == "range" else srv.submit_bpsw(r[1]))
        got = []
        for rid in ids:
            res = None
            for _ in range(600):
                res = srv.poll(rid, wait_ms=500)
                if res is not None:
                    break
            assert res is not None and res["status"] == 0
            got.append(res)
    for r, g in zip(reqs, got):
        if r[0] == "range":
            alone = engine.sieve_range(r[1], r[2])
            for k in ("pi", "max_gap", "gap_start", "twins"):
                assert g[k] == alone[k], (r, k)
        else:
            assert np.array_equal(g["verdicts"], engine.bpsw(r[1]))


def test_chunked_ranges_equal_alone(engine):
    """Ranges much longer than the serving chunk run in turns, interleaved with other requests,
    and join to the result of the whole range run alone."""
    import mathpub_b200 as mp
    reqs = _stream(29, 24, 24)
    with mp.Server(engine, streams=3, chunk=1 << 22) as srv:
        ids = [srv.submit_range(r[1], r[2]) if r[0] == "range" else srv.submit_bpsw(r[1]) for r in reqs]
        got = []
        for rid in ids:
            res = None
            for _ in range(600):
                res = srv.poll(rid, wait_ms=500)
                if res is not None:
                    break
            assert res is not None and res["status"] == 0
            got.append(res)
    nchunked = 0
    for r, g in zip(reqs, got):
        if r[0] == "range":
            nchunked += r[2] - r[1] > 1 << 22
            alone = engine.sieve_range(r[1], r[2])
            for k in ("pi", "max_gap", "gap_start", "twins"):
                assert g[k] == alone[k], (r, k)
        else:
            assert np.array_equal(g["verdicts"], engine.bpsw(r[1]))
    assert nchunked >= 5


def test_out_of_table_range_is_refused(engine):
    import mathpub_b200 as mp
    fresh = mp.Engine(0)             # its table is only as large as the server asks
    with mp.Server(fresh, streams=2, prime_limit=1 << 20) as srv:
        with pytest.raises(mp.MathpubError):
            srv.submit_range(10 ** 18, 10 ** 18 + 1000)
        rid = srv.submit_range(10 ** 9, 10 ** 9 + 100000)
        res = srv.poll(rid, wait_ms=60000)
        assert res["pi"] == engine.sieve_range(10 ** 9, 10 ** 9 + 100000)["pi"]
    fresh.close()


def test_close_with_requests_in_flight(engine):
    import mathpub_b200 as mp
    srv = mp.Server(engine, streams=2)
    for k in range(20):
        srv.submit_range(10 ** 12 + k * 2 ** 24, 10 ** 12 + (k + 1) * 2 ** 24)
    srv.close()                      # drains the queue, then stops the workers
