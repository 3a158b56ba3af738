"""Parity of the CUDA PM-basis and of the whole rank pipeline with the oracle
and with the reference's own golden outputs (bit-exact)."""
import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import synth

pytestmark = pytest.mark.gpu

P = 2013265921


def test_golden_reference_pm_basis_small_prime(ctx, golden):
    z = golden("pm_basis_ref.npz")
    for i in range(int(z["count"])):
        b, d, rank = (int(x) for x in z[f"c{i}_meta"])
        M, delta = rr.PM_Basis(z[f"c{i}_seq"], d, 3323, ctx)
        assert np.array_equal(M, z[f"c{i}_M"]), f"case {i} b={b} d={d}"
        assert np.array_equal(delta, z[f"c{i}_delta"]), f"case {i}"


@pytest.mark.parametrize("b,d", [(1, 1), (1, 64), (2, 2), (2, 256), (3, 40), (4, 8), (4, 128), (8, 32), (8, 64),
                                 (8, 1024), (16, 16), (16, 33), (16, 256), (32, 8), (32, 64)])
def test_random_sequences_vs_oracle(ctx, b, d):
    rng = np.random.default_rng(b * 1000 + d)
    dd = 1 << (d - 1).bit_length()
    seq = rng.integers(0, P, size=(b * (b + 1) // 2, dd + 2)).astype(np.uint32)
    M, delta = rr.PM_Basis(seq, d, P, ctx)
    Mo, do = oracle.pm_basis(seq, b, d, P)
    assert np.array_equal(M, Mo.astype(np.uint32))
    assert np.array_equal(delta, do)


def test_structured_sequence_with_dependent_rows(ctx):
    """A low-rank sequence exercises rows without pivots in every leaf."""
    b, d = 8, 128
    rng = np.random.default_rng(3)
    rowptr, col, val, m, n = synth.incidence(40, 30, seed=2)  # rank <= 30, tiny
    dr, dc = synth.preconditioners(m, n, P, 1)
    V = synth.random_vectors(b, n, P, 2)
    seq, L, _ = oracle.krylov(rowptr, col, val, m, n, P, dr, dc, V, 0, 2 * d)
    M, delta = rr.PM_Basis(seq, d, P, ctx)
    Mo, do = oracle.pm_basis(seq, b, d, P)
    assert np.array_equal(M, Mo.astype(np.uint32)) and np.array_equal(delta, do)
    assert rr.analyze_pm_basis(M, delta, P) == oracle.rank_from_basis(Mo, do, P)
    del rng


@pytest.mark.parametrize("p", [3323, 27644437, P])
@pytest.mark.parametrize("b", [1, 2, 4, 8])
def test_rank_of_matrix_txt(ctx, matrix_txt, p, b):
    rowptr, col, sval, m, n = matrix_txt
    val = (sval.astype(np.int64) % p).astype(np.uint32)
    a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
    assert rr.block_wiedemann_rank(a, b, p, seed=b, ctx=ctx) == 104


@pytest.mark.parametrize("b", [4, 8, 16])
def test_rank_known_by_construction(ctx, b):
    rowptr, col, val, m, n = synth.plain_single(n=1200, k=6, dep_rows=40, seed=b)
    dense = oracle.dense_rank_csr(rowptr, col, val, m, n, P)
    assert dense <= 1160
    a = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n)
    assert rr.block_wiedemann_rank(a, b, P, seed=7, ctx=ctx) == dense
    rp, cp = synth.preconditioners(m, n, P, 8)
    V = synth.random_vectors(b, n, P, 9)
    r_orc, _, _, _ = oracle.rank_pipeline(rowptr, col, val, m, n, P, rp, cp, V)
    assert rr.block_wiedemann_rank(a, b, P, row_precond=rp, col_precond=cp, v=V, ctx=ctx) == r_orc == dense


@pytest.mark.parametrize("b,d,count", [(2, 64, 3), (8, 256, 5), (16, 128, 4), (16, 64, 1), (3, 40, 2), (32, 16, 3)])
def test_batched_pm_basis_equals_single(ctx, b, d, count):
    """rr_pm_basis_batch (generators in lockstep) gives each sequence the
    generator rr_pm_basis gives it alone, bit for bit."""
    rng = np.random.default_rng(b * 31 + d)
    dd = 1 << (d - 1).bit_length()
    seqs = [rng.integers(0, P, size=(b * (b + 1) // 2, dd + 2)).astype(np.uint32) for _ in range(count)]
    got = rr.PM_Basis_batch(seqs, d, P, ctx)
    for s, (M, delta) in zip(seqs, got):
        M1, d1 = rr.PM_Basis(s, d, P, ctx)
        assert np.array_equal(M, M1) and np.array_equal(delta, d1)


def test_batched_pm_basis_small_prime_golden(ctx, golden):
    """The batched path on the reference's golden cases at p = 3323 (direct products)."""
    z = golden("pm_basis_ref.npz")
    by_shape = {}
    for i in range(int(z["count"])):
        b, d, _ = (int(x) for x in z[f"c{i}_meta"])
        by_shape.setdefault((b, d, z[f"c{i}_seq"].shape), []).append(i)
    for (b, d, _), idx in by_shape.items():
        got = rr.PM_Basis_batch([z[f"c{i}_seq"] for i in idx], d, 3323, ctx)
        for i, (M, delta) in zip(idx, got):
            assert np.array_equal(M, z[f"c{i}_M"]) and np.array_equal(delta, z[f"c{i}_delta"]), i


@pytest.mark.parametrize("b,d", [(8, 256), (16, 512), (16, 33), (4, 64)])
def test_cuda_core_contractions_equal_tensor_core(b, d):
    """The leaf residual updates and block-basis products on the CUDA cores
    (rr_ctx_set_pm_tensor_cores(ctx, 0)) give the tensor-core generator and the
    oracle's, bit for bit."""
    c = rr.Context(0)
    rng = np.random.default_rng(b * 7 + d)
    dd = 1 << (d - 1).bit_length()
    seq = rng.integers(0, P, size=(b * (b + 1) // 2, dd + 2)).astype(np.uint32)
    M_tc, d_tc = rr.PM_Basis(seq, d, P, c)
    c.set_pm_tensor_cores(False)
    M_cc, d_cc = rr.PM_Basis(seq, d, P, c)
    c.close()
    Mo, do = oracle.pm_basis(seq, b, d, P)
    assert np.array_equal(M_cc, M_tc) and np.array_equal(d_cc, d_tc)
    assert np.array_equal(M_cc, Mo.astype(np.uint32)) and np.array_equal(d_cc, do)
