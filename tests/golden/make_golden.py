"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Run from the repository root with a wilthoma/rust_rank checkout (read-only)
and the reference harness built from it:

    make -C oracle REF_DIR=<checkout>/cuda_test
    python tests/golden/make_golden.py --reference <checkout>

Fixtures written (all small):
  matrix_txt.npz      -- the reference's fixture cuda_test/matrix.txt as CSR
                         (signed values), its SHA-256 and its dense rank.
  pm_basis_ref.npz    -- PM_Basis outputs (M, delta) and the estimated rank
                         from the reference's C++ PM-basis
                         (cuda_test/sigma_basis.h) at p = 3323 for seeded
                         random sequences and for the Krylov sequences of
                         matrix.txt.
  linalg_kat.npz      -- lsp_decomposition / matrix_inverse / modular_rank
                         outputs of the reference on the matrices of its own
                         unit tests (src/modular_linalg.rs:437-497).
The reference's C++ code is exact for these sizes (p^2 * len * 2b < 2^61)
and its unstable delta sort equals the stable sort for 2b <= 16.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rust_rank_b200 import synth  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")
P_SMALL = 3323


def read_sms_signed(path):
    rows, cols, vals = [], [], []
    header = None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) != 3 or line.startswith("%"):
                continue
            if header is None:
                header = (int(parts[0]), int(parts[1]))
                continue
            r, c, v = int(parts[0]), int(parts[1]), int(parts[2])
            if r <= 0 or c <= 0:
                continue
            rows.append(r - 1)
            cols.append(c - 1)
            vals.append(v)
    return header, np.array(rows), np.array(cols), np.array(vals)


def ref_pm(R, seq, b, d, p):
    nlen = seq.shape[1]
    dd = 1
    while dd < d:
        dd *= 2
    M = np.zeros((2 * b, 2 * b, dd + 1), np.uint64)
    delta = np.zeros(2 * b, np.int64)
    ln = C.c_int64()
    R.ref_pm_basis(np.ascontiguousarray(seq, np.uint64), b, nlen, nlen, d, p, M, delta, C.byref(ln))
    assert ln.value == dd + 1
    rank = R.ref_rank_from_basis(M, delta, b, ln.value, p)
    return M, delta, rank


def main():
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the wilthoma/rust_rank checkout")
    args = ap.parse_args()
    ref_fixture = os.path.join(args.reference, "cuda_test", "matrix.txt")
    R = oracle.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref.so missing: run `make -C oracle REF_DIR=<checkout>/cuda_test`")
    # --- matrix.txt
    raw = open(ref_fixture, "rb").read()
    (m, n), rows, cols, vals = read_sms_signed(ref_fixture)
    order = np.argsort(rows, kind="stable")
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum(np.bincount(rows, minlength=m))
    col = cols[order].astype(np.int32)
    sval = vals[order].astype(np.int32)
    ranks = {}
    for p in (P_SMALL, 27644437, 2013265921):
        v = (sval.astype(np.int64) % p).astype(np.uint32)
        ranks[p] = oracle.dense_rank_csr(rowptr, col, v, m, n, p)
    np.savez_compressed(os.path.join(OUT, "matrix_txt.npz"), m=m, n=n, rowptr=rowptr, col=col, val=sval,
                        sha256=hashlib.sha256(raw).hexdigest(),
                        primes=np.array(sorted(ranks)), dense_ranks=np.array([ranks[k] for k in sorted(ranks)]))
    # --- PM-basis cases
    cases = {}
    rng = np.random.default_rng(20240601)
    idx = 0
    for b in (2, 3, 4, 8):
        for d in (1, 2, 4, 8, 16, 32, 64):
            seq = rng.integers(0, P_SMALL, size=(b * (b + 1) // 2, d + 1 + int(rng.integers(1, 4)))).astype(np.uint32)
            M, delta, rank = ref_pm(R, seq, b, d, P_SMALL)
            cases[f"c{idx}_seq"] = seq
            cases[f"c{idx}_meta"] = np.array([b, d, rank], np.int64)
            cases[f"c{idx}_M"] = M.astype(np.uint32)
            cases[f"c{idx}_delta"] = delta
            idx += 1
    # Krylov sequences of matrix.txt (preconditioners and V from fixed seeds)
    v_mod = (sval.astype(np.int64) % P_SMALL).astype(np.uint32)
    for b in (2, 4, 8):
        rp, cp = synth.preconditioners(m, n, P_SMALL, 11)
        V = synth.random_vectors(b, n, P_SMALL, 12)
        rank_o, seq, _, _ = oracle.rank_pipeline(rowptr, col, v_mod, m, n, P_SMALL, rp, cp, V)
        L = seq.shape[1]
        d = 1
        while d <= L:
            d *= 2
        d //= 2
        M, delta, rank = ref_pm(R, seq, b, d, P_SMALL)
        cases[f"c{idx}_seq"] = np.ascontiguousarray(seq, np.uint32)
        cases[f"c{idx}_meta"] = np.array([b, d, rank], np.int64)
        cases[f"c{idx}_M"] = M.astype(np.uint32)
        cases[f"c{idx}_delta"] = delta
        cases[f"c{idx}_krylov"] = np.array([11, 12], np.int64)  # seeds of (preconditioners, V)
        idx += 1
    cases["count"] = np.array(idx)
    np.savez_compressed(os.path.join(OUT, "pm_basis_ref.npz"), **cases)
    # --- linear algebra known-answer tests (inputs from src/modular_linalg.rs:437-497)
    kat = {}
    lsp_inputs = [
        (101, [[2, 4, 6], [1, 3, 5], [0, 0, 1]]),
        (97, [[10, 20, 30, 40, 50], [5, 10, 15, 20, 25], [0, 1, 0, 1, 0], [1, 0, 1, 0, 1], [99, 99, 99, 99, 99]]),
    ]
    for i, (p, a) in enumerate(lsp_inputs):
        a = np.array(a, np.uint64)
        k = a.shape[0]
        L = np.zeros_like(a)
        S = np.zeros_like(a)
        P = np.zeros_like(a)
        R.ref_lsp(k, np.ascontiguousarray(a), p, L, S, P)
        kat[f"lsp{i}_p"] = np.array(p)
        kat[f"lsp{i}_a"] = a
        kat[f"lsp{i}_L"] = L
        kat[f"lsp{i}_S"] = S
        kat[f"lsp{i}_P"] = P
        kat[f"lsp{i}_rank"] = np.array(R.ref_modular_rank(k, k, np.ascontiguousarray(a), p))
    for i, (p, a) in enumerate([(97, [[2, 3, 1], [1, 1, 1], [3, 5, 2]]), (97, np.eye(4, dtype=np.int64).tolist())]):
        a = np.array(a, np.uint64)
        out = np.zeros_like(a)
        R.ref_matrix_inverse(a.shape[0], np.ascontiguousarray(a), p, out)
        kat[f"inv{i}_p"] = np.array(p)
        kat[f"inv{i}_a"] = a
        kat[f"inv{i}_out"] = out
    np.savez_compressed(os.path.join(OUT, "linalg_kat.npz"), **kat)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
