"""Rank service (rr_server_*): requests submitted while others run get exactly
the rank they get alone (rr_rank on the same inputs) and the dense rank,
whatever the admission limits, lanes and interleaving."""
import time

import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921


def _requests(seed, count, rmin, rmax, b):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(rmin), np.log(rmax))))
        n = max(3, int(m * rng.uniform(0.6, 1.0)))
        dfc = n // 20 + 1 if i % 3 == 0 else 0
        rowptr, col, val, m, n = synth.incidence_fast(m, n, 4, 12, dfc, P, seed * 1000 + i)
        dr, dc = synth.preconditioners(m, n, P, seed + 7 * i + 1)
        V = synth.random_vectors(b, n, P, seed + 7 * i + 2)
        reqs.append((rowptr, col, val, m, n, dr, dc, V))
    return reqs


@pytest.mark.parametrize("b,lanes,max_active", [(8, 3, 4), (16, 4, 64), (4, 1, 1)])
def test_served_ranks_equal_alone_and_dense(ctx, b, lanes, max_active):
    reqs = _requests(11 + b, 10, 60, 1500, b)
    srv = rr.Server(b, P, lanes=lanes, workers=3, max_active=max_active, chunk_apps=16)
    ids = []
    rng = np.random.default_rng(5)
    for r in reqs:  # staggered arrivals: later requests join while earlier ones run
        ids.append(srv.submit(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]))
        time.sleep(float(rng.exponential(0.002)))
    got = [srv.result(i, timeout=120.0)[0] for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    for k, (rowptr, col, val, m, n, dr, dc, V) in enumerate(reqs):
        alone = rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(rowptr, col, val, m, n), b, P, dr, dc, V, ctx=ctx)
        assert got[k] == alone, (k, m, n, got[k], alone)
        assert got[k] == oracle.dense_rank_csr(rowptr, col, val, m, n, P), (k, m, n)


def test_server_admission_by_memory_budget(ctx):
    """A budget that admits about one request at a time still completes all of
    them with the same ranks; a request that can never fit is refused."""
    b = 8
    reqs = _requests(3, 5, 200, 400, b)
    srv = rr.Server(b, P, lanes=2, workers=2, hbm_budget=1_600_000)
    ids = [srv.submit(*r[:3], r[3], r[4], *r[5:]) for r in reqs]
    got = [srv.result(i, timeout=120.0)[0] for i in ids]
    for k, (rowptr, col, val, m, n, dr, dc, V) in enumerate(reqs):
        assert got[k] == rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(rowptr, col, val, m, n), b, P, dr, dc, V,
                                                 ctx=ctx)
    big = synth.incidence_fast(200000, 150000, 4, 12, 0, P, 9)
    dr, dc = synth.preconditioners(200000, 150000, P, 1)
    V = synth.random_vectors(b, 150000, P, 2)
    with pytest.raises(rr.RRError) as e:
        srv.submit(*big[:3], big[3], big[4], dr, dc, V)
    assert e.value.status == 3  # RR_ENOMEM
    srv.close()


def test_server_wait_times_out_on_host(ctx):
    """rr_server_wait with a short limit returns RR_ETIMEOUT (a host-side wait;
    the request still completes afterwards)."""
    b = 16
    rowptr, col, val, m, n = synth.incidence_fast(20000, 15000, 4, 12, 0, P, 4)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    srv = rr.Server(b, P)
    rid = srv.submit(rowptr, col, val, m, n, dr, dc, V)
    with pytest.raises(rr.RRError) as e:
        srv.result(rid, timeout=0.0)
    assert e.value.status == 5  # RR_ETIMEOUT
    rank, lat = srv.result(rid, timeout=120.0)
    assert rank == rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(rowptr, col, val, m, n), b, P, dr, dc, V, ctx=ctx)
    assert lat > 0
    srv.close()
