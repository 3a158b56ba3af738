"""Parity with the oracle at the benchmark sizes and at the hardest primes.

* the plain single-matrix workload in full (20,000 x 20,000, 6 entries per
  row, 500 dependent rows, b = 8, max_nlen = 8192 by the rule of
  src/main.rs:497-504): whole sequence, generator, rank;
* the PM-basis stage alone at b = 16, d = 2^14;
* the large Zipf matrix (2,000,000 x 1,500,000, 12 entries per row) at b = 16
  and 32: the first 64 sequence terms and the block after them;
* primes where the engine's arithmetic is tightest: p = 2^31 - 1 (largest
  accepted) and p = 1431655777, the first prime above 2^32 / 3, where
  c32 = 2^32 mod p is within 35 of p (the fold bound's worst case); and the
  reference's own small primes (3323, 2731, 1223), whose products go through
  the multi-prime CRT path.
All comparisons are bit-exact.
"""
import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921
P_MAX = 2147483647          # 2^31 - 1
P_TIGHT = 1431655777        # first prime above 2^32 / 3: 2^32 mod p = p - 35


def gpu_sequence(ctx, dm, V, rp, cp, max_nlen):
    ks = rr.KrylovStream(dm, V, rp, cp, 0)
    b = V.shape[0]
    seq = np.zeros((b * (b + 1) // 2, max_nlen + 1), np.uint32)
    L = ks.advance(max_nlen, seq)
    curv = ks.get_curv()
    ks.close()
    return seq[:, :L], curv


@pytest.mark.slow
def test_plain_single_matrix_full_pipeline(ctx):
    rowptr, col, val, m, n = synth.plain_single(n=20000, k=6, dep_rows=500, p=P, seed=43)
    b = 8
    rp, cp = synth.preconditioners(m, n, P, 5)
    V = synth.random_vectors(b, n, P, 6)
    max_nlen = rr.default_max_nlen(m, n, b)
    assert max_nlen == 8192
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    seq, curv = gpu_sequence(ctx, dm, V, rp, cp, max_nlen)
    s_orc, L, cv_orc = oracle.krylov(rowptr, col, val, m, n, P, rp, cp, V, 0, max_nlen)
    assert seq.shape[1] == L == max_nlen + 1
    assert np.array_equal(seq, s_orc)
    assert np.array_equal(curv, cv_orc)
    d = 8192
    M, delta = rr.PM_Basis(seq, d, P, ctx)
    Mo, do = oracle.pm_basis(s_orc, b, d, P)
    assert np.array_equal(M, Mo.astype(np.uint32)) and np.array_equal(delta, do)
    rank = rr.analyze_pm_basis(M, delta, P)
    assert rank == oracle.rank_from_basis(Mo, do, P)
    # the whole pipeline through rr_rank gives the same rank
    assert rr.block_wiedemann_rank(dm, b, P, row_precond=rp, col_precond=cp, v=V, ctx=ctx) == rank
    # 500 rows are combinations of others: rank <= 19,500
    assert rank == m - 500
    dm.close()


@pytest.mark.slow
def test_pm_basis_b16_d16384(ctx):
    b, d = 16, 1 << 14
    rng = np.random.default_rng(14)
    seq = rng.integers(0, P, size=(b * (b + 1) // 2, d + 1)).astype(np.uint32)
    M, delta = rr.PM_Basis(seq, d, P, ctx)
    Mo, do = oracle.pm_basis(seq, b, d, P)
    assert np.array_equal(M, Mo.astype(np.uint32)) and np.array_equal(delta, do)


@pytest.fixture(scope="module")
def zipf_full():
    return synth.zipf_large(p=P, seed=44)


@pytest.mark.slow
@pytest.mark.parametrize("b", [16, 32])
def test_zipf_full_first_64_terms(ctx, zipf_full, b):
    rowptr, col, val, m, n = zipf_full
    rp, cp = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(P, ctx)
    seq, curv = gpu_sequence(ctx, dm, V, rp, cp, 64)
    dm.close()
    s_orc, L, cv_orc = oracle.krylov(rowptr, col, val, m, n, P, rp, cp, V, 0, 64)
    assert seq.shape[1] == L == 65  # S_0 plus 32 applications of B
    assert np.array_equal(seq, s_orc)
    assert np.array_equal(curv, cv_orc)


@pytest.mark.parametrize("p", [P_MAX, P_TIGHT])
@pytest.mark.parametrize("b", [1, 5, 8, 16, 32])
def test_krylov_worst_case_primes(ctx, matrix_txt, p, b):
    rowptr, col, sval, m, n = matrix_txt
    val = (sval.astype(np.int64) % p).astype(np.uint32)
    rp, cp = synth.preconditioners(m, n, p, b + 1)
    V = synth.random_vectors(b, n, p, b + 2)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(p, ctx)
    seq, curv = gpu_sequence(ctx, dm, V, rp, cp, 24)
    dm.close()
    s_orc, _, cv_orc = oracle.krylov(rowptr, col, val, m, n, p, rp, cp, V, 0, 24)
    assert np.array_equal(seq, s_orc) and np.array_equal(curv, cv_orc)


@pytest.mark.parametrize("p", [P_MAX, P_TIGHT])
@pytest.mark.parametrize("b", [4, 16])
def test_krylov_heavy_rows_worst_case_primes(ctx, p, b):
    """Full-range values (worst case for the lazy sums) with rows long enough
    for the chunked path and every value equal to p - 1 in one dense row."""
    rng = np.random.default_rng(p % 1000 + b)
    m, n = 2500, 1800
    rows = []
    for r in range(m):
        if r % 500 == 3:
            c = np.arange(n)
        else:
            c = np.unique(np.concatenate([rng.choice(n, size=6), [5, 777]]))
        rows.append(c)
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.integers(1, p, size=col.size).astype(np.uint32)
    val[rowptr[3]:rowptr[4]] = p - 1
    rp = np.full(m, p - 1, np.uint32)
    cp = synth.preconditioners(m, n, p, 3)[1]
    V = np.full((b, n), p - 1, np.uint32)
    dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(p, ctx)
    seq, curv = gpu_sequence(ctx, dm, V, rp, cp, 8)
    dm.close()
    s_orc, _, cv_orc = oracle.krylov(rowptr, col, val, m, n, p, rp, cp, V, 0, 8)
    assert np.array_equal(seq, s_orc) and np.array_equal(curv, cv_orc)


@pytest.mark.parametrize("p,b,d", [(P_MAX, 16, 256), (P_MAX, 8, 1024), (P_TIGHT, 16, 256), (P_TIGHT, 4, 2048),
                                   (3323, 16, 4096), (2731, 16, 4096), (1223, 8, 4096), (27644437, 8, 512)])
def test_pm_basis_primes_without_ntt(ctx, p, b, d):
    """Primes whose p - 1 has no large power of two: the products are exact
    integer products over two or three NTT primes, combined by CRT."""
    rng = np.random.default_rng(p % 997 + d)
    seq = rng.integers(0, p, size=(b * (b + 1) // 2, d + 1)).astype(np.uint32)
    M, delta = rr.PM_Basis(seq, d, p, ctx)
    Mo, do = oracle.pm_basis(seq, b, d, p)
    assert np.array_equal(M, Mo.astype(np.uint32)) and np.array_equal(delta, do)


@pytest.mark.parametrize("p", [3323, P_TIGHT])
def test_batched_pm_basis_crt_equals_single(ctx, p):
    b, d = 8, 512
    rng = np.random.default_rng(p % 101)
    seqs = [rng.integers(0, p, size=(b * (b + 1) // 2, d + 1)).astype(np.uint32) for _ in range(3)]
    got = rr.PM_Basis_batch(seqs, d, p, ctx)
    for s, (M, delta) in zip(seqs, got):
        Mo, do = oracle.pm_basis(s, b, d, p)
        assert np.array_equal(M, Mo.astype(np.uint32)) and np.array_equal(delta, do)


@pytest.mark.parametrize("p", [3323, 2731])
def test_rank_pipeline_reference_primes(ctx, p):
    """The reference's working primes end to end: rank of a matrix with known
    deficit, against the oracle pipeline on the same preconditioners."""
    rowptr, col, val, m, n = synth.plain_single(n=3000, k=6, dep_rows=100, p=p, seed=p)
    b = 8
    rp, cp = synth.preconditioners(m, n, p, 11)
    V = synth.random_vectors(b, n, p, 12)
    a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
    r_gpu = rr.block_wiedemann_rank(a, b, p, row_precond=rp, col_precond=cp, v=V, ctx=ctx)
    r_orc, _, _, _ = oracle.rank_pipeline(rowptr, col, val, m, n, p, rp, cp, V)
    assert r_gpu == r_orc
    assert r_gpu <= m - 100
