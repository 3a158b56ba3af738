"""Host entry points around the generator (no GPU): the generator test of
src/blockbmtest.rs:445-461 and the scalar Berlekamp-Massey call surface of
src/block_berlekamp_massey.rs:104-131, against plain-Python restatements."""
import warnings

import numpy as np
import pytest

import rust_rank_b200 as rr

P = 2013265921


def py_is_generating_poly(poly, seq, p):
    """The reference loop, line by line (src/blockbmtest.rs:450-460)."""
    k, N, n = len(poly), len(seq), poly[0].shape[0]
    for l in range(N - k):
        s = np.zeros((n, n), dtype=object)
        for i in range(k):
            s = (s + seq[l + i].astype(object).dot(poly[i].astype(object))) % p
        if np.any(s != 0):
            return False
    return True


def py_massey(s, p):
    """Massey (1969), big integers."""
    C, B, L, m, b = [1], [1], 0, 1, 1
    for j in range(len(s)):
        d = s[j]
        for i in range(1, L + 1):
            d += C[i] * s[j - i]
        d %= p
        if d == 0:
            m += 1
            continue
        coef = d * pow(b, p - 2, p) % p
        T = list(C)
        C = C + [0] * max(0, len(B) + m - len(C))
        for i, x in enumerate(B):
            C[i + m] = (C[i + m] - coef * x) % p
        if 2 * L <= j:
            L, B, b, m = j + 1 - L, T, d, 1
        else:
            m += 1
    return [int(x) for x in (C + [0] * (L + 1))[: L + 1]], L


def recurrence_holds(conn, s, p):
    L = len(conn) - 1
    return all(sum(int(conn[i]) * int(s[j - i]) for i in range(L + 1)) % p == 0 for j in range(L, len(s)))


def test_bm_known_answers():
    fib = [0, 1]
    for _ in range(30):
        fib.append((fib[-1] + fib[-2]) % P)
    assert rr.berlekamp_massey(fib, P).tolist() == [1, P - 1, P - 1]  # 1 - x - x^2
    a = 123456789
    geo = [pow(a, j, P) for j in range(12)]
    assert rr.berlekamp_massey(geo, P).tolist() == [1, P - a]
    assert rr.berlekamp_massey([0] * 10, P).tolist() == [1]
    assert rr.berlekamp_massey([], P).tolist() == [1]
    # an impulse at position 3 has linear complexity 4
    assert len(rr.berlekamp_massey([0, 0, 0, 1], P)) == 5


@pytest.mark.parametrize("p", [3323, P])
@pytest.mark.parametrize("order", [1, 3, 8, 20])
def test_bm_recovers_random_recurrences(p, order):
    rng = np.random.default_rng(order * 7 + p % 1000)
    taps = [int(x) for x in rng.integers(0, p, size=order)]
    taps[-1] = taps[-1] or 1
    s = [int(x) for x in rng.integers(0, p, size=order)]
    for j in range(order, 2 * order + 16):
        s.append(sum(taps[i] * s[j - 1 - i] for i in range(order)) % p)
    conn = rr.berlekamp_massey(s, p)
    ref, L = py_massey(s, p)
    assert conn.tolist() == ref
    assert recurrence_holds(conn, s, p)
    assert L <= order
    if L == order:  # 2L terms or more determine the recurrence
        assert conn.tolist() == [1] + [(p - t) % p for t in taps]


def test_bm_matches_restatement_on_random_sequences():
    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 30, 61):
        s = [int(x) for x in rng.integers(0, 97, size=n)]
        conn = rr.berlekamp_massey(s, 97)
        assert conn.tolist() == py_massey(s, 97)[0]
        assert recurrence_holds(conn, s, 97)


def test_block_bm_call_surface():
    seq = [[1, 2, 4, 8, 16, 32], [5, 5, 5, 5, 5, 5]]
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        out = rr.block_berlekamp_massey(seq[:1], 1, 1, P)
    assert out.dtype == np.uint64 and out.tolist() == [1, P - 2]
    with pytest.warns(UserWarning):
        assert rr.block_berlekamp_massey(seq, 2, 2, P).tolist() == [1, P - 2]


def generated_sequence(rng, n, k, N, p):
    """poly with poly[k-1] = I and a sequence it generates by construction."""
    poly = rng.integers(0, p, size=(k, n, n), dtype=np.int64)
    poly[k - 1] = np.eye(n, dtype=np.int64)
    seq = [rng.integers(0, p, size=(n, n), dtype=np.int64) for _ in range(k - 1)]
    for l in range(N - k + 1):
        acc = np.zeros((n, n), dtype=object)
        for i in range(k - 1):
            acc = (acc + seq[l + i].astype(object).dot(poly[i].astype(object))) % p
        seq.append(((-acc) % p).astype(np.int64))
    return poly, np.array(seq, dtype=np.int64)


@pytest.mark.parametrize("p", [3323, P])
def test_is_generating_poly(p):
    rng = np.random.default_rng(11)
    n, k, N = 3, 4, 40
    poly, seq = generated_sequence(rng, n, k, N, p)
    assert py_is_generating_poly(list(poly), list(seq), p)
    assert rr.is_generating_poly(poly, seq, p)
    bad = seq.copy()
    bad[25, 1, 2] = (bad[25, 1, 2] + 1) % p
    assert not py_is_generating_poly(list(poly), list(bad), p)
    assert not rr.is_generating_poly(poly, bad, p)
    # the last term is outside every window of the reference's loop
    last = seq.copy()
    last[-1, 0, 0] = (last[-1, 0, 0] + 1) % p
    assert rr.is_generating_poly(poly, last, p) == py_is_generating_poly(list(poly), list(last), p)
    # random polynomials and sequences: both agree (almost always False)
    for _ in range(3):
        q = rng.integers(0, p, size=(2, n, n))
        s = rng.integers(0, p, size=(6, n, n))
        assert rr.is_generating_poly(q, s, p) == py_is_generating_poly(list(q), list(s), p)
    # N == k: no window, vacuously generating; N < k: an error
    assert rr.is_generating_poly(poly, seq[:k], p)
    with pytest.raises(rr.RRError):
        rr.is_generating_poly(poly, seq[: k - 1], p)
