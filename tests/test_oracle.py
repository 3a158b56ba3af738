"""The CPU oracle pinned against the reference: golden vectors produced by the
reference's own C++ PM-basis, the reference's unit-test inputs, its fixture
matrix and exact big-integer arithmetic.  No GPU needed."""
import numpy as np
import pytest

import oracle
from rust_rank_b200 import synth

P = 2013265921
P_SMALL = 3323


def test_matrix_txt_fixture_dense_rank(golden, matrix_txt):
    z = golden("matrix_txt.npz")
    rowptr, col, sval, m, n = matrix_txt
    assert (m, n, rowptr[-1]) == (182, 168, 1173)
    for p, r in zip(z["primes"], z["dense_ranks"]):
        v = (sval.astype(np.int64) % int(p)).astype(np.uint32)
        assert oracle.dense_rank_csr(rowptr, col, v, m, n, int(p)) == r == 104


def test_pm_basis_matches_reference_golden(golden):
    z = golden("pm_basis_ref.npz")
    for i in range(int(z["count"])):
        b, d, rank = (int(x) for x in z[f"c{i}_meta"])
        M, delta = oracle.pm_basis(z[f"c{i}_seq"], b, d, P_SMALL)
        assert np.array_equal(M.astype(np.uint32), z[f"c{i}_M"]), f"case {i}"
        assert np.array_equal(delta, z[f"c{i}_delta"]), f"case {i}"
        r = oracle.rank_from_basis(M, delta, P_SMALL)
        if r >= 0:  # the reference's unsigned formula is meaningless below degree 2
            assert r == rank, f"case {i}"


def test_krylov_sequences_of_matrix_txt_reproduce_reference_generator(golden, matrix_txt):
    """Sequences stored with the golden PM-basis cases are regenerated bit-exactly."""
    z = golden("pm_basis_ref.npz")
    rowptr, col, sval, m, n = matrix_txt
    v = (sval.astype(np.int64) % P_SMALL).astype(np.uint32)
    seen = 0
    for i in range(int(z["count"])):
        if f"c{i}_krylov" not in z:
            continue
        b, d, rank = (int(x) for x in z[f"c{i}_meta"])
        s1, s2 = (int(x) for x in z[f"c{i}_krylov"])
        rp, cp = synth.preconditioners(m, n, P_SMALL, s1)
        V = synth.random_vectors(b, n, P_SMALL, s2)
        r, seq, M, delta = oracle.rank_pipeline(rowptr, col, v, m, n, P_SMALL, rp, cp, V)
        assert np.array_equal(seq, z[f"c{i}_seq"])
        assert r == rank == 104
        seen += 1
    assert seen == 3


def test_linalg_known_answers(golden):
    z = golden("linalg_kat.npz")
    for i in range(2):
        p = int(z[f"lsp{i}_p"])
        a = z[f"lsp{i}_a"]
        L, S, perm = oracle.lsp(a, p)
        assert np.array_equal(L, z[f"lsp{i}_L"]) and np.array_equal(S, z[f"lsp{i}_S"])
        Pm = np.zeros_like(a)
        Pm[np.arange(len(perm)), perm] = 1
        assert np.array_equal(Pm, z[f"lsp{i}_P"])
        recon = (L.astype(object) @ S.astype(object) @ Pm.astype(object)) % p
        assert np.array_equal(recon.astype(np.uint64), a % p)
        assert oracle.modular_rank(a, p) == int(z[f"lsp{i}_rank"])
    for i in range(2):
        p = int(z[f"inv{i}_p"])
        assert np.array_equal(oracle.matrix_inverse(z[f"inv{i}_a"], p), z[f"inv{i}_out"])


def test_modinv_all_residues_mod_97():
    # src/modular_linalg.rs:500-507
    for a in range(1, 97):
        inv = oracle.matrix_inverse(np.array([[a]], np.uint64), 97)
        assert (a * int(inv[0, 0])) % 97 == 1


@pytest.mark.parametrize("n", [16, 256, 4096])
def test_ntt_roundtrip_and_dft(n):
    # src/ntt.rs:283-294 plus a direct DFT check
    rng = np.random.default_rng(n)
    a = rng.integers(0, P, size=n, dtype=np.uint64)
    f = oracle.ntt(a, False, P)
    assert np.array_equal(oracle.ntt(f, True, P), a)
    if n <= 256:
        g = oracle.generator(P)
        assert g == 31
        w = pow(g, (P - 1) // n, P)
        direct = [sum(int(a[j]) * pow(w, j * k, P) for j in range(n)) % P for k in range(n)]
        assert [int(x) for x in f] == direct


def test_poly_mat_mul_ntt_matches_schoolbook():
    # src/poly_mat_mul.rs:339-363
    rng = np.random.default_rng(7)
    a = rng.integers(0, P, size=(3, 4, 70), dtype=np.uint64)
    b = rng.integers(0, P, size=(4, 2, 90), dtype=np.uint64)
    c = oracle.poly_mat_mul(a, b, P, 5, 80)
    ref = np.zeros((3, 2, 70 + 75 - 1), dtype=object)
    for i in range(3):
        for j in range(2):
            for r in range(4):
                ref[i, j] += np.convolve(a[i, r].astype(object), b[r, j, 5:80].astype(object))
    assert np.array_equal(c, (ref % P).astype(np.uint64))


def _bigint_sequence(rowptr, col, val, m, n, p, dr, dc, V, L):
    A = np.zeros((m, n), dtype=object)
    for r in range(m):
        for k in range(rowptr[r], rowptr[r + 1]):
            A[r, col[k]] += int(val[k])
    Dr = np.diag([int(x) for x in dr]).astype(object)
    Dc = np.diag([int(x) for x in dc]).astype(object)
    B = (Dc @ A.T @ Dr @ A @ Dc) % p
    W = V.T.astype(object)
    out = []
    Bt = np.eye(n, dtype=object)
    for _ in range(L):
        S = (W.T @ Bt @ W) % p
        out.append(S)
        Bt = (Bt @ B) % p
    return out


@pytest.mark.parametrize("p", [P_SMALL, P])
def test_krylov_matches_big_integer_definition(p):
    rng = np.random.default_rng(p % 1000)
    m, n, b, L = 9, 7, 3, 9
    dense = rng.integers(0, p, size=(m, n)) * (rng.random((m, n)) < 0.5)
    rowptr = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.int64)
    rr_, cc = np.nonzero(dense)
    col = cc.astype(np.int32)
    val = dense[rr_, cc].astype(np.uint32)
    dr, dc = synth.preconditioners(m, n, p, 3)
    V = synth.random_vectors(b, n, p, 4)
    seq, length, _ = oracle.krylov(rowptr, col, val, m, n, p, dr, dc, V, 0, L - 1)
    assert length == L
    ref = _bigint_sequence(rowptr, col, val, m, n, p, dr, dc, V, L)
    iu = np.triu_indices(b)
    for t in range(L):
        assert [int(x) for x in seq[:, t]] == [int(x) for x in ref[t][iu]]


def test_krylov_resume_equals_one_shot():
    p = P
    rowptr, col, val, m, n = synth.incidence(40, 30, seed=5, p=p)
    dr, dc = synth.preconditioners(m, n, p, 1)
    V = synth.random_vectors(4, n, p, 2)
    full, L, cv_full = oracle.krylov(rowptr, col, val, m, n, p, dr, dc, V, 0, 16)
    part, L1, cv = oracle.krylov(rowptr, col, val, m, n, p, dr, dc, V, 0, 6)
    assert L1 == 7
    # a fresh start ends at max_nlen + 1 terms; a resume targets the length itself
    rest, L2, cv2 = oracle.krylov(rowptr, col, val, m, n, p, dr, dc, cv, L1, 17, seq=part)
    assert L2 == L == 17
    assert np.array_equal(rest, full) and np.array_equal(cv2, cv_full)


@pytest.mark.parametrize("p", [P_SMALL, 27644437, P])
@pytest.mark.parametrize("b", [1, 2, 4, 8])
def test_rank_pipeline_on_matrix_txt(matrix_txt, p, b):
    rowptr, col, sval, m, n = matrix_txt
    v = (sval.astype(np.int64) % p).astype(np.uint32)
    rp, cp = synth.preconditioners(m, n, p, 100 + b)
    V = synth.random_vectors(b, n, p, 200 + b)
    r, _, _, _ = oracle.rank_pipeline(rowptr, col, v, m, n, p, rp, cp, V)
    assert r == 104


def test_live_reference_harness_if_built():
    """When oracle/_ref was built (reference present), compare on fresh cases too."""
    import ctypes as C

    R = oracle.ref_lib()
    if R is None:
        pytest.skip("reference harness not built here")
    rng = np.random.default_rng(99)
    for b in (2, 5, 8):
        for d in (3, 16, 100):
            nlen = (1 << (d - 1).bit_length()) + 3
            seq = rng.integers(0, P_SMALL, size=(b * (b + 1) // 2, nlen)).astype(np.uint32)
            M, delta = oracle.pm_basis(seq, b, d, P_SMALL)
            Mr = np.zeros_like(M)
            dr = np.zeros_like(delta)
            ln = C.c_int64()
            R.ref_pm_basis(np.ascontiguousarray(seq, np.uint64), b, nlen, nlen, d, P_SMALL, Mr, dr, C.byref(ln))
            assert np.array_equal(M, Mr) and np.array_equal(delta, dr)


@pytest.mark.parametrize("b,nlen", [(2, 45), (3, 70), (4, 33)])
def test_pm_basis_reads_only_first_d_plus_1_terms(b, nlen):
    """PM_Basis(seq, d) depends on the first d + 1 terms only (M_Basis uses
    coefficient 0 and every product of _PM_Basis is truncated to d + 1
    coefficients, src/sigma_basis.rs:198,205).  The batched engine and the
    rank service rely on this to solve generators of equal order d together
    whatever their sequence lengths."""
    p = 2013265921
    rng = np.random.default_rng(b * 1000 + nlen)
    seq = rng.integers(0, p, size=(b * (b + 1) // 2, nlen), dtype=np.int64).astype(np.uint32)
    d = 1
    while d <= nlen:
        d *= 2
    d //= 2
    M_full, delta_full = oracle.pm_basis(seq, b, d, p)
    M_cut, delta_cut = oracle.pm_basis(seq[:, : d + 1], b, d, p)
    assert np.array_equal(M_full, M_cut) and np.array_equal(delta_full, delta_cut)
    # a change beyond term d changes nothing (term d itself is not read
    # either: the deepest leaf of the second half sees coefficient d - 1); a
    # change at term d - 1 does
    other = seq.copy()
    other[:, d:] = rng.integers(0, p, size=(other.shape[0], nlen - d), dtype=np.int64).astype(np.uint32)
    M_o, _ = oracle.pm_basis(other, b, d, p)
    assert np.array_equal(M_full, M_o)
    other[0, d - 1] = (int(other[0, d - 1]) + 1) % p
    M_d, _ = oracle.pm_basis(other, b, d, p)
    assert not np.array_equal(M_full, M_d)
