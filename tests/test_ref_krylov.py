"""The Krylov sequence pinned by the reference itself.

tests/golden/ref_krylov_matrix_txt.npz holds sequences made by the reference's
own CUDA Krylov program (cuda_test/cuvseq_int.cu, built unchanged for sm_100a
and run by tests/golden/make_ref_krylov.py) on its fixture cuda_test/matrix.txt
at p = 3323, with random preconditioners and starting blocks injected through a
.wdm checkpoint of length 0.  The oracle (CPU) and the engine (GPU, through the
C ABI) must reproduce every term and the final block exactly.
"""
import os

import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_krylov_matrix_txt.npz")


def _cases(golden, matrix_txt):
    z = golden("ref_krylov_matrix_txt.npz")
    p = int(z["p"])
    rowptr, col, sval, m, n = matrix_txt
    val = (sval.astype(np.int64) % p).astype(np.uint32)
    out = []
    for b in z["cases"]:
        k = f"b{int(b)}"
        out.append((int(b), p, rowptr, col, val, m, n, z[k + "_row_precond"], z[k + "_col_precond"], z[k + "_V"],
                    z[k + "_seq"], z[k + "_curv"]))
    return out


def test_fixture_shapes(golden, matrix_txt):
    for b, p, rowptr, col, val, m, n, rp, cp, V, seq, curv in _cases(golden, matrix_txt):
        assert p == 3323
        assert seq.shape[0] == b * (b + 1) // 2 and seq.shape[1] % 2 == 1
        assert rp.shape == (m,) and cp.shape == (n,) and V.shape == (b, n) and curv.shape == (b, n)
        assert (rp > 0).all() and (cp > 0).all() and (seq < p).all()


def test_oracle_reproduces_the_reference_sequence(golden, matrix_txt):
    for b, p, rowptr, col, val, m, n, rp, cp, V, seq, curv in _cases(golden, matrix_txt):
        L = seq.shape[1]
        got, Lo, cv = oracle.krylov(rowptr, col, val, m, n, p, rp, cp, V, 0, L - 1)
        assert Lo == L
        assert np.array_equal(got, seq), f"b={b}"
        assert np.array_equal(cv, curv), f"b={b}"


@pytest.mark.gpu
def test_engine_reproduces_the_reference_sequence(ctx, golden, matrix_txt):
    for b, p, rowptr, col, val, m, n, rp, cp, V, seq, curv in _cases(golden, matrix_txt):
        L = seq.shape[1]
        dm = rr.CsrMatrix.from_arrays(rowptr, col, val, m, n).to_device(p, ctx)
        ks = rr.KrylovStream(dm, V, rp, cp, 0)
        out = np.zeros((b * (b + 1) // 2, L + 1), np.uint32)
        assert ks.advance(L - 1, out) == L
        assert np.array_equal(out[:, :L], seq), f"b={b}"
        assert np.array_equal(ks.get_curv(), curv), f"b={b}"
        ks.close()
        dm.close()
