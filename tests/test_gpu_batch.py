"""Batched engine (rr_batch_*): every matrix of a stacked batch gets exactly the
sequence, generator and rank it gets alone -- checked against the oracle's
Krylov sequence, the single-matrix GPU pipeline and dense ranks."""
import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921


def _mixed_batch(seed, count=9, rmin=40, rmax=900):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(rmin), np.log(rmax))))
        n = max(3, int(m * rng.uniform(0.6, 1.0)))
        dfc = n // 20 + 1 if i % 3 == 0 else 0
        mats.append(synth.incidence_fast(m, n, 3, 10, dfc, P, seed * 100 + i))
    # one wide matrix and one with empty rows and columns
    mats.append(synth.incidence_fast(120, 300, 2, 5, 0, P, seed + 7))
    rowptr, col, val, m, n = synth.incidence_fast(200, 150, 1, 3, 0, P, seed + 8)
    lens = np.diff(rowptr)
    lens[::7] = 0  # rows 0, 7, 14, ... empty
    mask = np.repeat(lens > 0, np.diff(rowptr))
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    mats.append((rp, col[mask], val[mask], m, n))
    return mats


def _inputs(mats, b, seed):
    drs, dcs, vs = [], [], []
    for i, (_, _, _, m, n) in enumerate(mats):
        dr, dc = synth.preconditioners(m, n, P, seed + 10 * i + 1)
        drs.append(dr)
        dcs.append(dc)
        vs.append(synth.random_vectors(b, n, P, seed + 10 * i + 2))
    return drs, dcs, vs


@pytest.mark.parametrize("b", [3, 4, 8, 16, 32])
def test_batch_sequences_match_oracle(ctx, b):
    mats = _mixed_batch(b)
    drs, dcs, vs = _inputs(mats, b, 5)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    bt.krylov()
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        L = rr.default_max_nlen(m, n, b)
        ref, Lr, _ = oracle.krylov(rowptr, col, val, m, n, P, drs[i], dcs[i], vs[i], 0, L)
        got = bt.sequence(i)
        assert got.shape[1] == Lr, (i, got.shape, Lr)
        assert np.array_equal(got, ref[:, :Lr]), f"matrix {i} ({m}x{n}) differs"
    bt.close()


@pytest.mark.parametrize("b,workers", [(8, 1), (8, 4), (16, 3)])
def test_batch_ranks_match_single_and_dense(ctx, b, workers):
    mats = _mixed_batch(100 + b, rmin=120)
    drs, dcs, vs = _inputs(mats, b, 9)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    ranks = bt.ranks(workers)  # Krylov and generators overlapped
    bt.close()
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
        single = rr.block_wiedemann_rank(a, b, P, drs[i], dcs[i], vs[i], ctx=ctx)
        assert ranks[i] == single, (i, ranks[i], single)
        assert ranks[i] == oracle.dense_rank_csr(rowptr, col, val, m, n, P), (i, m, n)


def test_batch_ranks_after_krylov(ctx):
    """Generators from a batch whose sequences were computed first (no
    overlap) equal the overlapped run."""
    b = 16
    mats = _mixed_batch(77, count=6, rmin=120)
    drs, dcs, vs = _inputs(mats, b, 3)
    a = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    a.krylov()
    r1 = a.ranks(2)
    a.close()
    c = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    r2 = c.ranks(5)
    c.close()
    assert np.array_equal(r1, r2)


def test_batch_single_matrix_and_order(ctx):
    """A batch of one, and a batch given longest-first, keep the caller's order."""
    b = 8
    mats = _mixed_batch(5, count=4, rmin=120)[::-1]
    drs, dcs, vs = _inputs(mats, b, 1)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    ranks = bt.ranks(2)
    bt.close()
    for i in range(len(mats)):
        one = rr.Batch([mats[i]], b, P, [drs[i]], [dcs[i]], [vs[i]], ctx)
        assert one.ranks(1)[0] == ranks[i]
        one.close()


def test_batch_rejects_bad_input(ctx):
    b = 4
    mats = _mixed_batch(2, count=2)
    drs, dcs, vs = _inputs(mats, b, 1)
    bad = list(mats)
    rowptr, col, val, m, n = bad[0]
    col = col.copy()
    col[0] = n  # out of range
    bad[0] = (rowptr, col, val, m, n)
    with pytest.raises(rr.RRError):
        rr.Batch(bad, b, P, drs, dcs, vs, ctx)
    dcs2 = [d.copy() for d in dcs]
    dcs2[1][0] = 0  # preconditioners must be units
    with pytest.raises(rr.RRError):
        rr.Batch(mats, b, P, drs, dcs2, vs, ctx)


@pytest.mark.slow
def test_batch_graph_complex_subset(ctx):
    """A 24-matrix slice of the graph-complex-like set (rows up to 20,000):
    batched ranks equal one-at-a-time ranks."""
    b = 16
    mats = synth.graph_complex_batch(nmat=24, rmin=1000, rmax=20000, seed=11)
    drs, dcs, vs = _inputs(mats, b, 21)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    ranks = bt.ranks(8)
    bt.close()
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
        assert ranks[i] == rr.block_wiedemann_rank(a, b, P, drs[i], dcs[i], vs[i], ctx=ctx), i


def test_batch_autotuner_shapes(ctx):
    """The autotuner picks, per phase of the Krylov loop, a grid of 1..4 CTAs
    per SM and the lanes each thread owns; phases start at increasing
    applications; results stay exact."""
    b = 8
    mats = _mixed_batch(31, count=7)
    drs, dcs, vs = _inputs(mats, b, 13)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    shapes = bt.tuning()
    assert len(shapes) >= 1 and shapes[0][0] == 0
    assert all(s1[0] > s0[0] for s0, s1 in zip(shapes, shapes[1:]))
    assert all(c % 148 == 0 and 148 <= c <= 4 * 148 for _, c in shapes) or all(c >= 1 for _, c in shapes)
    lanes = bt.tuning_shape()  # block shape beside the grid: 4 or 8 lanes per thread at padded width 8
    assert len(lanes) == len(shapes)
    assert all(lpt in (4, 8) and rows == 32 * lpt // 8 for lpt, rows in lanes)
    bt.krylov()
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        L = rr.default_max_nlen(m, n, b)
        ref, Lr, _ = oracle.krylov(rowptr, col, val, m, n, P, drs[i], dcs[i], vs[i], 0, L)
        assert np.array_equal(bt.sequence(i), ref[:, :Lr]), i
    bt.close()


def test_batch_with_heavy_rows_and_columns(ctx):
    """Matrices with rows and columns far above the chunking threshold (a dense
    row, a dense column) in the batch: sequences equal the oracle's."""
    b = 16
    rng = np.random.default_rng(77)
    mats = _mixed_batch(41, count=5)
    m, n = 900, 700
    rows = []
    for r in range(m):
        if r == 5:
            c = np.arange(n)  # dense row of A (a heavy row of the stack)
        else:
            c = np.unique(np.concatenate([rng.choice(n, size=4), [11]]))  # column 11 dense: heavy row of A^T
        rows.append(c)
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.integers(1, P, size=col.size).astype(np.uint32)
    mats.insert(2, (rowptr, col, val, m, n))
    drs, dcs, vs = _inputs(mats, b, 17)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    bt.krylov()
    for i, (rowptr, col, val, m, n) in enumerate(mats):
        L = rr.default_max_nlen(m, n, b)
        ref, Lr, _ = oracle.krylov(rowptr, col, val, m, n, P, drs[i], dcs[i], vs[i], 0, L)
        assert np.array_equal(bt.sequence(i), ref[:, :Lr]), i
    bt.close()


def test_grid_barrier_gives_up_and_context_survives(ctx):
    """The persistent launch's grid barrier: with every CTA arriving it passes;
    waiting for one CTA more than the grid has, every wait runs out after its
    limit and reports it, and the context keeps working."""
    import ctypes as C
    import time

    from rust_rank_b200 import _lib

    t = C.c_int32(-1)
    _lib.check(_lib.lib().rr_device_barrier_check(ctx.handle, 148, 148, 20, 1.0, C.byref(t)))
    assert t.value == 0
    t0 = time.perf_counter()
    _lib.check(_lib.lib().rr_device_barrier_check(ctx.handle, 148, 149, 3, 0.3, C.byref(t)))
    assert t.value == 1
    assert time.perf_counter() - t0 < 10
    # the context still runs work
    b = 4
    mats = _mixed_batch(5, count=3)
    drs, dcs, vs = _inputs(mats, b, 3)
    bt = rr.Batch(mats, b, P, drs, dcs, vs, ctx)
    bt.krylov()
    rowptr, col, val, m, n = mats[0]
    ref, Lr, _ = oracle.krylov(rowptr, col, val, m, n, P, drs[0], dcs[0], vs[0], 0, rr.default_max_nlen(m, n, b))
    assert np.array_equal(bt.sequence(0), ref[:, :Lr])
    bt.close()
