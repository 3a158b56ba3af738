"""Parity of the CUDA Krylov step with the oracle (bit-exact), through the C ABI."""
import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921


def gpu_sequence(ctx, rowptr, col, val, m, n, p, dr, dc, V, max_nlen, seq_len=0, prev=None):
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(p, ctx)
    ks = rr.KrylovStream(dm, V, dr, dc, seq_len)
    b = V.shape[0]
    seq = np.zeros((b * (b + 1) // 2, max(max_nlen, seq_len) + 2), np.uint32)
    if prev is not None:
        seq[:, : prev.shape[1]] = prev
    L = ks.advance(max_nlen, seq)
    return seq[:, :L], ks.get_curv(), ks


def check_against_oracle(ctx, rowptr, col, val, m, n, p, b, max_nlen, seed=0):
    dr, dc = synth.preconditioners(m, n, p, seed + 1)
    V = synth.random_vectors(b, n, p, seed + 2)
    s_gpu, cv_gpu, _ = gpu_sequence(ctx, rowptr, col, val, m, n, p, dr, dc, V, max_nlen)
    s_orc, L, cv_orc = oracle.krylov(rowptr, col, val, m, n, p, dr, dc, V, 0, max_nlen)
    assert s_gpu.shape[1] == L
    assert np.array_equal(s_gpu, s_orc)
    assert np.array_equal(cv_gpu, cv_orc)


@pytest.mark.parametrize("p", [3323, 27644437, P])
@pytest.mark.parametrize("b", [1, 2, 3, 4, 5, 8, 12, 16, 24, 32])
def test_matrix_txt(ctx, matrix_txt, p, b):
    rowptr, col, sval, m, n = matrix_txt
    val = (sval.astype(np.int64) % p).astype(np.uint32)
    check_against_oracle(ctx, rowptr, col, val, m, n, p, b, 20, seed=b)


@pytest.mark.parametrize("b", [4, 16, 32])
def test_heavy_rows_and_columns(ctx, b):
    """Dense rows of A and dense columns (rows of A^T longer than the split
    threshold) go through the chunked path."""
    rng = np.random.default_rng(b)
    m, n = 3000, 2000
    rows = []
    for r in range(m):
        if r % 997 == 5:
            c = np.sort(rng.choice(n, size=1500, replace=False))
        else:
            c = np.unique(np.concatenate([rng.choice(n, size=5), [7, 1234, 1999]]))
        rows.append(c)
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.integers(1, P, size=col.size).astype(np.uint32)
    check_against_oracle(ctx, rowptr, col, val, m, n, P, b, 10, seed=3)


def test_zipf_small(ctx):
    rowptr, col, val, m, n = synth.zipf_large(m=20000, n=15000, k=12, dup_rows=100, seed=9)
    check_against_oracle(ctx, rowptr, col, val, m, n, P, 16, 8, seed=4)


def test_empty_rows_columns_and_rectangular(ctx):
    rng = np.random.default_rng(1)
    m, n = 50, 80
    dense = rng.integers(1, P, size=(m, n)) * (rng.random((m, n)) < 0.05)
    dense[3] = 0
    dense[:, 10] = 0
    dense[:, 79] = 0
    rowptr = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.int64)
    r_, c_ = np.nonzero(dense)
    check_against_oracle(ctx, rowptr, c_.astype(np.int32), dense[r_, c_].astype(np.uint32), m, n, P, 6, 12)
    # transposed shape too
    dt = dense.T.copy()
    rowptr = np.concatenate([[0], np.cumsum((dt != 0).sum(1))]).astype(np.int64)
    r_, c_ = np.nonzero(dt)
    check_against_oracle(ctx, rowptr, c_.astype(np.int32), dt[r_, c_].astype(np.uint32), n, m, P, 6, 12)


def test_resume_from_checkpoint_state(ctx):
    rowptr, col, val, m, n = synth.incidence(400, 300, seed=5)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(8, n, P, 2)
    full, L, cv_full = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 16)
    part, L1, cv = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 6)
    s_gpu, cv_gpu, _ = gpu_sequence(ctx, rowptr, col, val, m, n, P, dr, dc, cv, 17, seq_len=L1, prev=part)
    assert np.array_equal(s_gpu, full) and np.array_equal(cv_gpu, cv_full)


def test_device_steps_fetch_and_next(ctx):
    rowptr, col, val, m, n = synth.incidence(500, 450, seed=6)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(16, n, P, 2)
    ref, L, _ = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 20)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    ks = rr.KrylovStream(dm, V, dr, dc, 0)
    ks.step_device(4)
    ks.step_device(6)
    assert len(ks) == 21
    out = np.zeros((136, 21), np.uint32)
    ks.fetch(0, 21, out)
    assert np.array_equal(out, ref)
    # VectorStream::next returns w_{k+1} (src/vectorstream.rs:58-69)
    ks2 = rr.KrylovStream(dm, V, dr, dc, 0)
    w1 = np.array(ks2.next())
    _, _, cv1 = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 2)
    assert np.array_equal(w1, cv1)


def test_main_loop_with_checkpoint(ctx, tmp_path):
    rowptr, col, val, m, n = synth.incidence(300, 200, seed=8)
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(4, n, P, 2)
    ref, L, cv_ref = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 64)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    ks = rr.KrylovStream(dm, V, dr, dc, 0)
    seq = np.zeros((10, 66), np.uint32)
    curv = V.copy()
    path = str(tmp_path / "m_4.wdm")
    L2 = rr.main_loop_s_mt2(ks, dr, dc, curv, V, seq, 0, 64, wdm_filename=path, theprime=P, chunk_terms=10)
    assert L2 == L == 65
    assert np.array_equal(seq[:, :L2], ref) and np.array_equal(curv, cv_ref)
    p, mm, nn, b, rp2, cp2, v2, cv2, seq2 = rr.load_wdm_file_sym(path)
    assert (p, mm, nn, b) == (P, m, n, 4) and np.array_equal(seq2, ref) and np.array_equal(cv2, cv_ref)


def test_invalid_arguments_fail_loudly(ctx):
    rowptr, col, val, m, n = synth.incidence(30, 20, seed=1)
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.from_arrays(rowptr, np.where(col == col[0], 25, col), val, m, n).to_device(P, ctx)
    assert e.value.status == 1
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(2013265923, ctx)
    assert e.value.status == 2
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    dr, dc = synth.preconditioners(m, n, P, 1)
    for b in (0, 33):
        with pytest.raises(rr.RRError):
            rr.KrylovStream(dm, np.zeros((b, n), np.uint32), dr, dc)
    dc0 = dc.copy()
    dc0[3] = 0
    with pytest.raises(rr.RRError):
        rr.KrylovStream(dm, np.zeros((2, n), np.uint32), dr, dc0)


def test_two_runs_are_identical(ctx):
    """Determinism of two GPU runs (the reference checks it for its GPU
    products, cuda_test/cupoly_mat_mul.h:638-690): sequence and generator of
    the same inputs, computed twice, are bit-identical (the arithmetic is
    exact, so no reduction order can change them)."""
    rowptr, col, val, m, n = synth.plain_single(n=3000, k=6, dep_rows=50, p=P, seed=17)
    b = 16
    dr, dc = synth.preconditioners(m, n, P, 18)
    V = synth.random_vectors(b, n, P, 19)
    L = rr.default_max_nlen(m, n, b)
    runs = []
    for _ in range(2):
        s, cv, ks = gpu_sequence(ctx, rowptr, col, val, m, n, P, dr, dc, V, L)
        ks.close()
        d = 1
        while d <= s.shape[1]:
            d *= 2
        d //= 2
        M, delta = rr.PM_Basis(s, d, P, ctx)
        runs.append((s, cv, M, delta))
    for a, b_ in zip(runs[0], runs[1]):
        assert np.array_equal(a, b_)
