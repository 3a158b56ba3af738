"""Sharding by matrix (rr_fleet_*, rr_batch_ranks_multi) and the device-side
matrix build.

The pool gives one GPU per run, so the multi-device paths run with the same
device listed more than once: two services (or two batches) share it, the
placement and routing logic runs as it would across GPUs, and every rank must
equal the single-matrix path's."""
import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921


def _mats(seed, count, rmin, rmax, b):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(rmin), np.log(rmax))))
        n = max(3, int(m * rng.uniform(0.6, 1.0)))
        rowptr, col, val, m, n = synth.incidence_fast(m, n, 3, 10, n // 25 if i % 3 == 0 else 0, P, seed * 100 + i)
        dr, dc = synth.preconditioners(m, n, P, seed + 5 * i + 1)
        V = synth.random_vectors(b, n, P, seed + 5 * i + 2)
        out.append((rowptr, col, val, m, n, dr, dc, V))
    return out


@pytest.mark.parametrize("devices", [[0], [0, 0], [0, 0, 0]])
def test_fleet_ranks_equal_alone(ctx, devices):
    b = 8
    reqs = _mats(21, 9, 80, 1200, b)
    fl = rr.Fleet(b, P, devices=devices, lanes=2, workers=2, chunk_apps=16, hbm_budget=64 << 20)
    ids = [fl.submit(*r[:3], r[3], r[4], *r[5:]) for r in reqs]
    got = [fl.result(i, timeout=120.0)[0] for i in ids]
    where = [fl.device_of(i) for i in ids]
    st = fl.stats()
    fl.close()
    assert st["completed"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert set(where) <= set(devices)
    for k, (rowptr, col, val, m, n, dr, dc, V) in enumerate(reqs):
        alone = rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(rowptr, col, val, m, n), b, P, dr, dc, V, ctx=ctx)
        assert got[k] == alone, (k, m, n)


def test_batch_ranks_multi_equal_single(ctx):
    b = 16
    mats = _mats(33, 12, 100, 3000, b)
    ranks, where = rr.batch_ranks_multi([x[:5] for x in mats], b, P, [x[5] for x in mats], [x[6] for x in mats],
                                        [x[7] for x in mats], devices=[0, 0], workers=2)
    assert set(where.tolist()) <= {0}
    for k, (rowptr, col, val, m, n, dr, dc, V) in enumerate(mats):
        alone = rr.block_wiedemann_rank(rr.CsrMatrix.from_arrays(rowptr, col, val, m, n), b, P, dr, dc, V, ctx=ctx)
        assert ranks[k] == alone, (k, m, n)


def test_device_build_rejects_bad_input(ctx):
    rowptr, col, val, m, n = synth.plain_single(n=300, k=5, dep_rows=10, p=P, seed=3)
    bad = col.copy()
    bad[77] = n
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.from_arrays(rowptr, bad, val, m, n).to_device(P, ctx)
    assert e.value.status == 1 and "entry 77" in str(e.value)
    badv = val.copy()
    badv[5] = P
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.from_arrays(rowptr, col, badv, m, n).to_device(P, ctx)
    assert e.value.status == 1 and "entry 5" in str(e.value)
    badp = rowptr.copy()
    badp[40] = badp[41] + 1
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.from_arrays(badp, col, val, m, n).to_device(P, ctx)
    assert e.value.status == 1 and "row 40" in str(e.value)


@pytest.mark.parametrize("b", [8, 16, 32])
def test_device_build_duplicates_empty_and_dense(ctx, b):
    """Duplicate entries in a row, empty rows and columns (the zero tail of
    both degree orders), a dense row and a dense column (chunked on both
    sides), at the widths of the fused, split and tcgen05 Gram forms: same
    sequence and block as the oracle."""
    rng = np.random.default_rng(9)
    m, n = 2100, 1700
    rows = []
    for r in range(m):
        if r == 17:
            c = np.arange(n - 60)  # the last 60 columns stay empty
        elif r % 11 == 0:
            c = np.array([], np.int64)
        else:
            c = np.concatenate([rng.choice(n - 100, size=4), [3, 3, 999]])  # duplicates of column 3
        rows.append(np.sort(c))
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.integers(0, P, size=col.size).astype(np.uint32)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    assert dm.max_nnzs() == (int(np.diff(rowptr).max()), int(np.bincount(col, minlength=n).max()))
    assert int((np.bincount(col, minlength=n) == 0).sum()) == 60
    ks = rr.KrylovStream(dm, V, dr, dc, 0)
    seq = np.zeros((b * (b + 1) // 2, 20), np.uint32)
    L = ks.advance(16, seq)
    s_orc, Lo, cv_orc = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 16)
    assert L == Lo and np.array_equal(seq[:, :L], s_orc)
    assert np.array_equal(ks.get_curv(), cv_orc)
