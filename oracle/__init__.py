"""CPU oracle for the block-Wiedemann rank path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/liboracle.so`` (the exact mod-p CPU restatement of
the reference algorithm in ``rr_oracle.cpp``) and, when it was built, to
``oracle/_ref/libref.so`` (the reference's own C++ PM-basis headers compiled
in place).  Only the tests, the smoke entry point and bench.py's CPU baseline
/ reference arm use this module; the engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i64 = C.c_int64
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    """Compile liboracle.so (and the reference harness when the reference is present)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_krylov.restype = _i64
        L.orc_krylov.argtypes = [_i64, _i64, _i64p, _i32p, _u32p, C.c_uint32, C.c_int, _u32p, _u32p, _u32p,
                                 _i64, _i64, _u32p, _i64]
        L.orc_op_create.restype = C.c_void_p
        L.orc_op_create.argtypes = [_i64, _i64, _i64p, _i32p, _u32p, C.c_uint32, C.c_int, _u32p, _u32p, _u32p]
        L.orc_op_step.restype = C.c_int
        L.orc_op_step.argtypes = [C.c_void_p, _u32p, _u32p]
        L.orc_op_destroy.restype = None
        L.orc_op_destroy.argtypes = [C.c_void_p]
        L.orc_lsp.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _u64p, _i32p]
        L.orc_matrix_inverse.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p]
        L.orc_modular_rank.restype = _i64
        L.orc_modular_rank.argtypes = [C.c_int, C.c_int, _u64p, C.c_uint64]
        L.orc_dense_rank_csr.restype = _i64
        L.orc_dense_rank_csr.argtypes = [_i64, _i64, _i64p, _i32p, _u32p, C.c_uint64]
        L.orc_poly_mat_mul.argtypes = [C.c_int, C.c_int, C.c_int, _i64, _i64, _u64p, _u64p, C.c_uint64, _i64,
                                       _i64, _u64p]
        L.orc_ntt.argtypes = [_u64p, _i64, C.c_int, C.c_uint64]
        L.orc_generator.restype = C.c_uint64
        L.orc_generator.argtypes = [C.c_uint64]
        L.orc_pm_basis.argtypes = [_u32p, C.c_int, _i64, _i64, _i64, C.c_uint32, _u64p, _i64p]
        L.orc_rank_from_basis.restype = _i64
        L.orc_rank_from_basis.argtypes = [_u64p, _i64p, C.c_int, _i64, C.c_uint64]
        L.orc_num_threads.restype = C.c_int
        L.orc_num_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference harness library, or None when it was not built here."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_pm_basis.argtypes = [_u64p, C.c_int, _i64, _i64, _i64, C.c_uint64, _u64p, _i64p, C.POINTER(_i64)]
        R.ref_rank_from_basis.restype = _i64
        R.ref_rank_from_basis.argtypes = [_u64p, _i64p, C.c_int, _i64, C.c_uint64]
        R.ref_lsp.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p, _u64p, _u64p]
        R.ref_matrix_inverse.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p]
        R.ref_modular_rank.restype = _i64
        R.ref_modular_rank.argtypes = [C.c_int, C.c_int, _u64p, C.c_uint64]
        R.ref_poly_mat_mul.argtypes = [C.c_int, C.c_int, C.c_int, _i64, _i64, _u64p, _u64p, C.c_uint64, _i64,
                                       _i64, _u64p, C.POINTER(_i64)]
        _REF = R
    return _REF


def set_threads(n: int) -> int:
    return lib().orc_num_threads(int(n))


# ---------------------------------------------------------------- Krylov
def krylov(rowptr, col, val, m, n, p, row_precond, col_precond, curv, seq_len, max_nlen, seq=None):
    """Krylov sequence as in src/main.rs:88-216.  Returns (seq [np][cap], new_len, curv)."""
    b = curv.shape[0]
    np_ = b * (b + 1) // 2
    cap = max(max_nlen + 1, seq_len + 1)
    out = np.zeros((np_, cap), np.uint32)
    if seq is not None:
        out[:, : seq.shape[1]] = seq[:, : min(seq.shape[1], cap)]
    cv = np.ascontiguousarray(curv, dtype=np.uint32).copy()
    new_len = lib().orc_krylov(m, n, np.ascontiguousarray(rowptr, np.int64), np.ascontiguousarray(col, np.int32),
                               np.ascontiguousarray(val, np.uint32), p, b,
                               np.ascontiguousarray(row_precond, np.uint32),
                               np.ascontiguousarray(col_precond, np.uint32), cv, seq_len, max_nlen, out, cap)
    if new_len < 0:
        raise ValueError("oracle krylov: bad arguments")
    return out[:, :new_len], new_len, cv


class KrylovOp:
    """One application of B at a time (for timing the CPU baseline)."""

    def __init__(self, rowptr, col, val, m, n, p, row_precond, col_precond, curv):
        self.b = curv.shape[0]
        self.np = self.b * (self.b + 1) // 2
        self.h = lib().orc_op_create(m, n, np.ascontiguousarray(rowptr, np.int64), np.ascontiguousarray(col, np.int32),
                                     np.ascontiguousarray(val, np.uint32), p, self.b,
                                     np.ascontiguousarray(row_precond, np.uint32),
                                     np.ascontiguousarray(col_precond, np.uint32),
                                     np.ascontiguousarray(curv, np.uint32))

    def step(self):
        g1 = np.zeros(self.np, np.uint32)
        g2 = np.zeros(self.np, np.uint32)
        lib().orc_op_step(self.h, g1, g2)
        return g1, g2

    def close(self):
        if self.h:
            lib().orc_op_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# ---------------------------------------------------------------- generator
def pm_basis(seq, b, d, p):
    """PM_Basis (src/sigma_basis.rs:9-54).  seq: [b(b+1)/2][nlen] -> (M [2b][2b][d'+1], delta [2b])."""
    seq = np.ascontiguousarray(seq, np.uint32)
    nlen = seq.shape[1]
    dd = 1
    while dd < d:
        dd *= 2
    M = np.zeros((2 * b, 2 * b, dd + 1), np.uint64)
    delta = np.zeros(2 * b, np.int64)
    rc = lib().orc_pm_basis(seq, b, nlen, nlen, d, p, M, delta)
    if rc != 0:
        raise ValueError(f"oracle pm_basis failed ({rc})")
    return M, delta


def rank_from_basis(M, delta, p):
    b = M.shape[0] // 2
    return int(lib().orc_rank_from_basis(np.ascontiguousarray(M, np.uint64), np.ascontiguousarray(delta, np.int64),
                                         b, M.shape[2], p))


def lsp(a, p):
    a = np.ascontiguousarray(a, np.uint64)
    m = a.shape[0]
    L = np.zeros_like(a)
    S = np.zeros_like(a)
    perm = np.zeros(m, np.int32)
    lib().orc_lsp(m, a, p, L, S, perm)
    return L, S, perm


def matrix_inverse(a, p):
    a = np.ascontiguousarray(a, np.uint64)
    out = np.zeros_like(a)
    if lib().orc_matrix_inverse(a.shape[0], a, p, out) != 0:
        raise ValueError("singular")
    return out


def modular_rank(a, p):
    a = np.ascontiguousarray(a, np.uint64)
    return int(lib().orc_modular_rank(a.shape[0], a.shape[1], a, p))


def dense_rank_csr(rowptr, col, val, m, n, p):
    r = lib().orc_dense_rank_csr(m, n, np.ascontiguousarray(rowptr, np.int64), np.ascontiguousarray(col, np.int32),
                                 np.ascontiguousarray(val, np.uint32), p)
    if r < 0:
        raise ValueError("matrix too large for the dense check")
    return int(r)


def poly_mat_mul(a, b, p, b_start=0, b_end=None):
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    m, n, la = a.shape
    _, k, lb = b.shape
    if b_end is None:
        b_end = lb + b_start
    lres = la + min(lb, b_end - b_start) - 1
    out = np.zeros((m, k, lres), np.uint64)
    lib().orc_poly_mat_mul(m, n, k, la, lb, a, b, p, b_start, b_end, out)
    return out


def ntt(a, invert, p):
    a = np.ascontiguousarray(a, np.uint64).copy()
    if lib().orc_ntt(a, a.shape[0], int(invert), p) != 0:
        raise ValueError("length not supported by p")
    return a


def generator(p):
    return int(lib().orc_generator(p))


def rank_pipeline(rowptr, col, val, m, n, p, row_precond, col_precond, V, max_nlen=None):
    """Krylov sequence + PM-basis + rank readout, driven like src/main.rs:497-606."""
    b = V.shape[0]
    if max_nlen is None:
        max_nlen = int(np.floor(2.0 * min(m, n) / b + 4.0))
        if b > 1:
            max_nlen = 1 << (max_nlen - 1).bit_length()
    seq, L, _ = krylov(rowptr, col, val, m, n, p, row_precond, col_precond, V, 0, max_nlen)
    d = 1
    while d <= L:
        d *= 2
    d //= 2
    M, delta = pm_basis(seq, b, d, p)
    return rank_from_basis(M, delta, p), seq, M, delta
