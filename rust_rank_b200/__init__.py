"""B200 block-Wiedemann rank engine: Python host layer over librr_b200.so.

Mirrors the reference's call surface for the rank path (wilthoma/rust_rank):

* ``CsrMatrix``            -- src/matrices.rs:53-64 (+ load_csr_matrix_from_sms, max_nnzs)
* ``KrylovStream``         -- src/vectorstream.rs:7-10 (VectorStream: next, fill_status)
* ``main_loop_s_mt2``      -- src/main.rs:88-216 (sequence S_t = V^T B^t V, checkpointing)
* ``PM_Basis``             -- src/sigma_basis.rs:9-54
* ``analyze_pm_basis``     -- src/sigma_basis.rs:71-152 + src/blockbmtest.rs:574-599 (returns the rank)
* ``save_wdm_file_sym`` / ``load_wdm_file_sym`` -- src/wdm_files.rs
* ``block_wiedemann_rank`` -- the driver of src/main.rs:463-606

All arithmetic runs in the CUDA library; nothing here computes on the CPU
beyond argument marshalling.
"""
from __future__ import annotations

import atexit
import ctypes as C
import sys
import time
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import RRError, check, lib, ptr  # noqa: F401

# Live handles by teardown order (states and batches, then matrices, then
# contexts): closed at interpreter exit before module teardown, so a handle is
# never destroyed after the context it lives on.
_LIVE = (weakref.WeakSet(), weakref.WeakSet(), weakref.WeakSet())


def _track(obj, level: int):
    _LIVE[level].add(obj)


@atexit.register
def _close_all():
    for group in _LIVE:
        for obj in list(group):
            try:
                obj.close()
            except Exception:
                pass


__all__ = ["Context", "CsrMatrix", "DeviceMatrix", "KrylovStream", "main_loop_s_mt2", "PM_Basis",
           "analyze_pm_basis", "block_wiedemann_rank", "save_wdm_file_sym", "load_wdm_file_sym",
           "default_max_nlen", "Batch", "Server", "RRError", "is_generating_poly", "berlekamp_massey",
           "block_berlekamp_massey"]

DEFAULT_PRIME = 2013265921


class Context:
    """One CUDA device and the stream all engine work is queued on."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().rr_ctx_create(device, C.byref(h)))
        self.handle = h
        _track(self, 2)
        self.device = device

    @property
    def stream(self) -> int:
        return lib().rr_ctx_stream(self.handle) or 0

    def set_pm_tensor_cores(self, enable: bool):
        """PM-basis contractions on the int8 tensor cores (True, default) or the CUDA cores (False)."""
        check(lib().rr_ctx_set_pm_tensor_cores(self.handle, 1 if enable else 0))

    def synchronize(self):
        check(lib().rr_ctx_synchronize(self.handle))

    def close(self):
        if self.handle:
            lib().rr_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT_CTX: Context | None = None


def default_context() -> Context:
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


@dataclass
class CsrMatrix:
    """Host CSR matrix over F_p (src/matrices.rs:53-64); values in [0, p)."""

    values: np.ndarray       # uint32
    col_indices: np.ndarray  # int32
    row_ptr: np.ndarray      # int64
    n_rows: int
    n_cols: int

    @staticmethod
    def from_arrays(rowptr, col, val, m, n) -> "CsrMatrix":
        return CsrMatrix(np.ascontiguousarray(val, np.uint32), np.ascontiguousarray(col, np.int32),
                         np.ascontiguousarray(rowptr, np.int64), int(m), int(n))

    @staticmethod
    def load_csr_matrix_from_sms(path: str, theprime: int) -> "CsrMatrix":
        """src/matrices.rs:662-732."""
        L = lib()
        m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        check(L.rr_sms_load(path.encode(), theprime, C.byref(m), C.byref(n), C.byref(nnz), None, None, None))
        rowptr = np.zeros(m.value + 1, np.int64)
        col = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros(max(nnz.value, 1), np.uint32)
        check(L.rr_sms_load(path.encode(), theprime, C.byref(m), C.byref(n), C.byref(nnz), ptr(rowptr), ptr(col),
                            ptr(val)))
        return CsrMatrix(val[: nnz.value], col[: nnz.value], rowptr, m.value, n.value)

    def max_nnzs(self):
        """src/matrices.rs:842-860."""
        rows = np.diff(self.row_ptr)
        cols = np.bincount(self.col_indices, minlength=self.n_cols)
        return int(rows.max(initial=0)), int(cols.max(initial=0))

    def to_device(self, theprime: int, ctx: Context | None = None) -> "DeviceMatrix":
        return DeviceMatrix(self, theprime, ctx or default_context())


class DeviceMatrix:
    """A CSR matrix resident on the GPU (degree-ordered copy plus its transpose)."""

    def __init__(self, a: CsrMatrix, theprime: int, ctx: Context):
        self.ctx = ctx
        self.p = int(theprime)
        self.n_rows, self.n_cols = a.n_rows, a.n_cols
        h = C.c_void_p()
        check(lib().rr_matrix_create(ctx.handle, a.n_rows, a.n_cols, ptr(a.row_ptr), ptr(a.col_indices),
                                     ptr(a.values), self.p, C.byref(h)))
        self.handle = h
        _track(self, 1)

    def max_nnzs(self):
        r, c = C.c_int64(), C.c_int64()
        check(lib().rr_matrix_max_nnzs(self.handle, C.byref(r), C.byref(c)))
        return r.value, c.value

    def close(self):
        if getattr(self, "handle", None):
            lib().rr_matrix_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KrylovStream:
    """VectorStream (src/vectorstream.rs:7-10) for B = D_c A^T D_r A D_c on the GPU.

    ``next()`` returns w_{k+1} = B w_k as ``b`` host vectors, like the
    reference's worker threads; ``main_loop_s_mt2`` instead keeps the vectors
    on the device and only brings back the sequence terms.
    """

    def __init__(self, a: DeviceMatrix, curv, row_precond, col_precond, seq_len: int = 0):
        curv = np.ascontiguousarray(curv, np.uint32)
        self.b = curv.shape[0]
        self.n = a.n_cols
        self.a = a
        self.row_precond = np.ascontiguousarray(row_precond, np.uint32)
        self.col_precond = np.ascontiguousarray(col_precond, np.uint32)
        h = C.c_void_p()
        check(lib().rr_krylov_create(a.handle, self.b, ptr(self.row_precond), ptr(self.col_precond), ptr(curv),
                                     int(seq_len), C.byref(h)))
        self.handle = h
        _track(self, 0)

    def __len__(self) -> int:
        v = C.c_int64()
        check(lib().rr_krylov_length(self.handle, C.byref(v)))
        return v.value

    def next(self):
        check(lib().rr_krylov_step_device(self.handle, 1))
        return list(self.get_curv())

    def fill_status(self) -> str:
        """src/vectorstream.rs:7-10: one line on the stream's state."""
        buf = C.create_string_buffer(256)
        check(lib().rr_krylov_fill_status(self.handle, buf, 256))
        return buf.value.decode()

    def get_curv(self, out: np.ndarray | None = None) -> np.ndarray:
        """The current block w_k, [b][n] in the caller's column order.  `out`: a
        C-contiguous uint32 [b][n] array to write into (e.g. pinned host memory)."""
        if out is None:
            out = np.empty((self.b, self.n), np.uint32)
        elif out.dtype != np.uint32 or out.shape != (self.b, self.n) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous uint32 array of shape {(self.b, self.n)}")
        check(lib().rr_krylov_get_curv(self.handle, ptr(out)))
        return out

    def advance(self, max_nlen: int, seq: np.ndarray, report=None, chunk_terms: int = 0) -> int:
        """Extend the sequence up to max_nlen terms (see rr_krylov_advance).

        ``report(len, target_len, elapsed_s, terms_per_s) -> bool`` (optional)
        is called after every chunk of ``chunk_terms`` terms, like the
        reference's report_progress (src/main.rs:57-85); returning True stops
        the advance there (to save a checkpoint, src/main.rs:186-202)."""
        new_len = C.c_int64()
        if report is None:
            check(lib().rr_krylov_advance(self.handle, int(max_nlen), ptr(seq), seq.shape[1], C.byref(new_len)))
            return new_len.value
        errors = []

        def cb(_user, length, target, elapsed, rate):
            try:
                return 1 if report(int(length), int(target), float(elapsed), float(rate)) else 0
            except Exception as e:  # stop and re-raise on the Python side
                errors.append(e)
                return 1

        fn = _lib.PROGRESS_FN(cb)
        check(lib().rr_krylov_advance_report(self.handle, int(max_nlen), ptr(seq), seq.shape[1], int(chunk_terms), fn,
                                             None, C.byref(new_len)))
        if errors:
            raise errors[0]
        return new_len.value

    def step_device(self, n_apps: int):
        check(lib().rr_krylov_step_device(self.handle, int(n_apps)))

    def fetch(self, lo: int, hi: int, seq: np.ndarray):
        check(lib().rr_krylov_fetch(self.handle, int(lo), int(hi), ptr(seq), seq.shape[1]))

    def bytes_per_application(self) -> float:
        v = C.c_double()
        check(lib().rr_krylov_bytes_per_application(self.handle, C.byref(v)))
        return v.value

    def phase_bytes(self):
        v = (C.c_double * 2)()
        check(lib().rr_krylov_phase_bytes(self.handle, v))
        return v[0], v[1]

    def profile(self, n_apps: int):
        """Mean device ms per application: (pass over A, chunks of A^T, pass over A^T)."""
        v = (C.c_double * 3)()
        check(lib().rr_krylov_profile(self.handle, int(n_apps), v))
        return v[0], v[1], v[2]

    def launch_count(self) -> int:
        v = C.c_int64()
        check(lib().rr_krylov_launch_count(self.handle, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "handle", None):
            lib().rr_krylov_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_max_nlen(m: int, n: int, num_v: int) -> int:
    """Sequence length rule of src/main.rs:497-504."""
    max_nlen = int(np.floor(np.float32(2.0) * np.float32(min(m, n)) / np.float32(num_v) + np.float32(4.0)))
    if num_v > 1:
        max_nlen = 1 << (max_nlen - 1).bit_length()
    return max_nlen


def report_progress(length: int, target: int, elapsed: float, rate: float, num_v: int, out=None) -> None:
    """The progress line of src/main.rs:57-85: terms done, elapsed time, throughput, time remaining."""
    remaining = (target - length) / rate if rate > 0 else float("inf")
    print(f"\rProgress: {length}/{target} | Elapsed: {int(elapsed)}s | Throughput: {rate:.1f}/s "
          f"(total {rate * num_v:.1f}/s) | Remaining: {remaining:.1f}s", end="", flush=True, file=out or sys.stdout)


def main_loop_s_mt2(stream: KrylovStream, row_precond, col_precond, curv, v, seq: np.ndarray, seq_len: int,
                    max_nlen: int, wdm_filename: str | None = None, theprime: int = DEFAULT_PRIME,
                    save_after: float = 200.0, chunk_terms: int = 1 << 14, report_every: float | None = None) -> int:
    """src/main.rs:88-216.  ``seq`` is [b(b+1)/2][>= max_nlen + 1] and holds
    ``seq_len`` terms; returns the new length.  The current block is written
    back into ``curv`` and, every ``save_after`` seconds, saved to the .wdm
    file (src/main.rs:186-202); with ``report_every`` (seconds) a progress line
    is printed like the reference's report_progress (src/main.rs:57-85)."""
    last_save = time.time()
    last_report = [0.0]
    b = stream.b

    def report(length, target, elapsed, rate):
        if report_every is not None and elapsed - last_report[0] >= report_every:
            report_progress(length, target, elapsed, rate, b)
            last_report[0] = elapsed
        # stop the advance when a checkpoint is due
        return bool(wdm_filename) and time.time() - last_save > save_after

    L = seq_len
    while True:
        L = stream.advance(max_nlen, seq, report=report, chunk_terms=chunk_terms)
        done = max_nlen - L < 2
        if wdm_filename:
            curv[:] = stream.get_curv()
            save_wdm_file_sym(wdm_filename, stream.a.n_rows, stream.n, theprime, row_precond, col_precond, v, curv,
                              seq[:, :L])
            last_save = time.time()
        if done:
            break
    if report_every is not None:
        print(file=sys.stdout)
    curv[:] = stream.get_curv()
    return L


def PM_Basis(seq: np.ndarray, d: int, seqprime: int, ctx: Context | None = None):
    """src/sigma_basis.rs:9-54 -> (M [2b][2b][d+1], delta [2b])."""
    ctx = ctx or default_context()
    seq = np.ascontiguousarray(seq, np.uint32)
    nn, nlen = seq.shape
    b = int((np.sqrt(8 * nn + 1) - 1) // 2)
    if b * (b + 1) // 2 != nn:
        raise ValueError("Sequence length does not match square matrix size")
    dd = 1
    while dd < d:
        dd *= 2
    M = np.zeros((2 * b, 2 * b, dd + 1), np.uint32)
    delta = np.zeros(2 * b, np.int64)
    check(lib().rr_pm_basis(ctx.handle, ptr(seq), nlen, b, nlen, dd, seqprime, ptr(M), ptr(delta)))
    return M, delta


def PM_Basis_batch(seqs, d: int, seqprime: int, ctx: Context | None = None):
    """PM_Basis of several sequences of equal shape solved in lockstep
    (rr_pm_basis_batch); returns [(M, delta)] in order."""
    ctx = ctx or default_context()
    seqs = [np.ascontiguousarray(s, np.uint32) for s in seqs]
    nn, nlen = seqs[0].shape
    b = int((np.sqrt(8 * nn + 1) - 1) // 2)
    if b * (b + 1) // 2 != nn or any(s.shape != seqs[0].shape for s in seqs):
        raise ValueError("sequences must share one square block size and length")
    dd = 1
    while dd < d:
        dd *= 2
    Ms = [np.zeros((2 * b, 2 * b, dd + 1), np.uint32) for _ in seqs]
    ds = [np.zeros(2 * b, np.int64) for _ in seqs]
    cnt = len(seqs)
    arr = lambda xs: (C.c_void_p * cnt)(*[x.ctypes.data for x in xs])  # noqa: E731
    strides = np.full(cnt, nlen, np.int64)
    check(lib().rr_pm_basis_batch(ctx.handle, cnt, arr(seqs), ptr(strides), b, nlen, dd, seqprime, arr(Ms), arr(ds)))
    return list(zip(Ms, ds))


def analyze_pm_basis(basis: np.ndarray, delta: np.ndarray, p: int) -> int:
    """src/sigma_basis.rs:71-152 -> src/blockbmtest.rs:574-599; returns the estimated rank."""
    basis = np.ascontiguousarray(basis, np.uint32)
    delta = np.ascontiguousarray(delta, np.int64)
    r = C.c_int64()
    check(lib().rr_rank_from_basis(ptr(basis), ptr(delta), basis.shape[0] // 2, basis.shape[2], p, C.byref(r)))
    return r.value


def is_generating_poly(poly, seq, p: int) -> bool:
    """src/blockbmtest.rs:445-461: whether sum_{i<k} seq[l+i] @ poly[i] == 0 mod p for
    every l in [0, N - k).  poly: k matrices n x n, seq: N matrices n x n (residues)."""
    poly = np.ascontiguousarray(np.asarray(poly, dtype=np.int64) % p, np.uint32)
    seq = np.ascontiguousarray(np.asarray(seq, dtype=np.int64) % p, np.uint32)
    if poly.ndim != 3 or seq.ndim != 3 or poly.shape[1:] != seq.shape[1:] or poly.shape[1] != poly.shape[2]:
        raise ValueError("poly and seq must be stacks of equal square matrices")
    ok = C.c_int32()
    check(lib().rr_is_generating_poly(ptr(poly), poly.shape[0], ptr(seq), seq.shape[0], poly.shape[1], p,
                                      C.byref(ok)))
    return bool(ok.value)


def berlekamp_massey(seq, p: int) -> np.ndarray:
    """Shortest linear recurrence of a scalar sequence mod p (Massey's algorithm):
    the connection polynomial [1, c_1, ..., c_L] with sum_i c_i seq[j - i] = 0 for j >= L."""
    s = np.ascontiguousarray(np.asarray(seq, dtype=np.int64) % p, np.uint32)
    conn = np.zeros(s.size + 1, np.uint32)
    L = C.c_int64()
    check(lib().rr_berlekamp_massey(ptr(s), s.size, p, ptr(conn), C.byref(L)))
    return conn[: L.value + 1].copy()


def block_berlekamp_massey(seq, num_u: int, num_v: int, p: int) -> np.ndarray:
    """The call surface of src/block_berlekamp_massey.rs:104-131: only block width 1
    is implemented (as in the reference, which warns and uses seq[0] otherwise); the
    scalar sequence seq[0] goes to berlekamp_massey."""
    if num_u > 1 or num_v > 1:
        import warnings

        warnings.warn("Matrix Berlekamp-Massey is not implemented; using the first sequence only", stacklevel=2)
    return berlekamp_massey(np.asarray(seq[0]), p).astype(np.uint64)


def block_wiedemann_rank(a: CsrMatrix | DeviceMatrix, num_v: int, theprime: int = DEFAULT_PRIME,
                         row_precond=None, col_precond=None, v=None, max_nlen: int = 0, seed: int | None = None,
                         ctx: Context | None = None) -> int:
    """The rank path of src/main.rs:463-606 in one call (rr_rank)."""
    from . import synth

    dm = a if isinstance(a, DeviceMatrix) else a.to_device(theprime, ctx)
    rng_seed = 0 if seed is None else seed
    if row_precond is None or col_precond is None:
        row_precond, col_precond = synth.preconditioners(dm.n_rows, dm.n_cols, theprime, rng_seed + 1)
    if v is None:
        v = synth.random_vectors(num_v, dm.n_cols, theprime, rng_seed + 2)
    row_precond = np.ascontiguousarray(row_precond, np.uint32)
    col_precond = np.ascontiguousarray(col_precond, np.uint32)
    v = np.ascontiguousarray(v, np.uint32)
    r = C.c_int64()
    check(lib().rr_rank(dm.handle, num_v, ptr(row_precond), ptr(col_precond), ptr(v), int(max_nlen), C.byref(r)))
    return r.value


class Batch:
    """Many matrices ranked together (rr_batch_*): one Krylov launch per pass
    for the whole stack, generators solved concurrently as sequences finish.

    ``mats`` is a list of (rowptr, col, val, m, n); ``row_preconds``,
    ``col_preconds`` and ``vs`` give each matrix's preconditioners and its
    b x n block V.  Every matrix gets the same sequence, generator and rank
    as :func:`block_wiedemann_rank` on it alone."""

    def __init__(self, mats, num_v: int, theprime: int, row_preconds, col_preconds, vs, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.n = len(mats)
        self.b = int(num_v)
        keep = []

        def arr(xs, dt):
            out = [np.ascontiguousarray(x, dt) for x in xs]
            keep.extend(out)
            return (C.c_void_p * self.n)(*[a.ctypes.data for a in out])

        m = np.array([int(x[3]) for x in mats], np.int64)
        n = np.array([int(x[4]) for x in mats], np.int64)
        rp = arr([x[0] for x in mats], np.int64)
        cl = arr([x[1] for x in mats], np.int32)
        vl = arr([x[2] for x in mats], np.uint32)
        rpc = arr(row_preconds, np.uint32)
        cpc = arr(col_preconds, np.uint32)
        vv = arr(vs, np.uint32)
        h = C.c_void_p()
        check(lib().rr_batch_create(self.ctx.handle, self.n, ptr(m), ptr(n), rp, cl, vl, int(theprime), self.b, rpc,
                                    cpc, vv, C.byref(h)))
        self.handle = h
        _track(self, 0)

    def krylov(self):
        check(lib().rr_batch_krylov(self.handle))

    def sequence(self, i: int) -> np.ndarray:
        L = C.c_int64()
        check(lib().rr_batch_sequence(self.handle, i, None, 0, C.byref(L)))
        seq = np.zeros((self.b * (self.b + 1) // 2, L.value), np.uint32)
        check(lib().rr_batch_sequence(self.handle, i, ptr(seq), L.value, C.byref(L)))
        return seq

    def ranks(self, workers: int = 8) -> np.ndarray:
        out = np.zeros(self.n, np.int64)
        check(lib().rr_batch_ranks(self.handle, int(workers), ptr(out)))
        return out

    def tuning(self):
        """[(first application, CTAs)] per phase of the Krylov loop, as the autotuner chose them."""
        k = C.c_int32(0)
        check(lib().rr_batch_tuning(self.handle, C.byref(k), None, None))
        ctas = np.zeros(k.value, np.int32)
        first = np.zeros(k.value, np.int64)
        check(lib().rr_batch_tuning(self.handle, C.byref(k), ptr(ctas), ptr(first)))
        return [(int(a), int(c)) for a, c in zip(first, ctas)]

    def tuning_shape(self):
        """[(lanes per thread, rows per warp batch)] per phase, as the autotuner chose them."""
        k = C.c_int32(0)
        check(lib().rr_batch_tuning_shape(self.handle, C.byref(k), None, None))
        lanes = np.zeros(k.value, np.int32)
        rows = np.zeros(k.value, np.int32)
        check(lib().rr_batch_tuning_shape(self.handle, C.byref(k), ptr(lanes), ptr(rows)))
        return [(int(a), int(b)) for a, b in zip(lanes, rows)]

    def info(self):
        r, c, z, a = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().rr_batch_info(self.handle, C.byref(r), C.byref(c), C.byref(z), C.byref(a)))
        return {"rows": r.value, "cols": c.value, "nnz": z.value, "max_apps": a.value}

    def close(self):
        if getattr(self, "handle", None):
            lib().rr_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Rank service (rr_server_*): requests are submitted as they arrive,
    admitted by device-memory footprint, their Krylov steps interleaved on
    several streams and their generators solved by worker threads.  Every
    request gets exactly the rank :func:`block_wiedemann_rank` gives on the
    same inputs."""

    def __init__(self, num_v: int, theprime: int = DEFAULT_PRIME, lanes: int = 4, workers: int = 4,
                 max_active: int = 64, chunk_apps: int = 64, hbm_budget: int = 0, device: int = 0):
        from ._lib import ServerConfig

        cfg = ServerConfig(int(num_v), int(theprime), int(lanes), int(workers), int(max_active), int(chunk_apps),
                           int(hbm_budget))
        h = C.c_void_p()
        check(lib().rr_server_create(device, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.b = int(num_v)
        _track(self, 0)

    def submit(self, rowptr, col, val, m: int, n: int, row_precond, col_precond, v) -> int:
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.uint32)
        rp = np.ascontiguousarray(row_precond, np.uint32)
        cp = np.ascontiguousarray(col_precond, np.uint32)
        v = np.ascontiguousarray(v, np.uint32)
        if rp.size != m or cp.size != n or v.shape != (self.b, n):
            raise ValueError("preconditioner or block shapes do not match the matrix")
        rid = C.c_uint64()
        check(lib().rr_server_submit(self.handle, m, n, ptr(rowptr), ptr(col), ptr(val), ptr(rp), ptr(cp), ptr(v),
                                     C.byref(rid)))
        return rid.value

    def result(self, rid: int, timeout: float = -1.0):
        """(rank, latency in ms) of request ``rid``, waiting up to ``timeout`` seconds (< 0: no limit)."""
        r, lat = C.c_int64(), C.c_double()
        check(lib().rr_server_wait(self.handle, rid, float(timeout), C.byref(r), C.byref(lat)))
        return r.value, lat.value

    def stats(self):
        a, b = C.c_int64(), C.c_int64()
        p50, p99, rps = C.c_double(), C.c_double(), C.c_double()
        check(lib().rr_server_stats(self.handle, C.byref(a), C.byref(b), C.byref(p50), C.byref(p99), C.byref(rps)))
        return {"submitted": a.value, "completed": b.value, "p50_ms": p50.value, "p99_ms": p99.value,
                "ranks_per_s": rps.value}

    def close(self):
        if getattr(self, "handle", None):
            lib().rr_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(m: int, n: int, nnz: int, num_v: int) -> int:
    """Device bytes a matrix and its Krylov state hold while resident (rr_footprint)."""
    v = C.c_uint64()
    check(lib().rr_footprint(int(m), int(n), int(nnz), int(num_v), C.byref(v)))
    return v.value


def place_by_footprint(footprints, dev_free):
    """Placement of independent matrices on devices (rr_place_by_footprint):
    largest first, each onto the device with the most room left.  Returns
    (device index per item, bytes placed per device)."""
    fp = np.ascontiguousarray(footprints, np.uint64)
    fr = np.ascontiguousarray(dev_free, np.uint64)
    where = np.zeros(fp.size, np.int32)
    load = np.zeros(fr.size, np.uint64)
    check(lib().rr_place_by_footprint(fp.size, ptr(fp), fr.size, ptr(fr), ptr(where), ptr(load)))
    return where, load


def _pointer_arrays(keep, xs, dt):
    out = [np.ascontiguousarray(x, dt) for x in xs]
    keep.extend(out)
    return (C.c_void_p * len(out))(*[a.ctypes.data for a in out])


def batch_ranks_multi(mats, num_v: int, theprime: int, row_preconds, col_preconds, vs, devices, workers: int = 8):
    """Ranks of many matrices over several GPUs (rr_batch_ranks_multi): each
    matrix is placed whole on one device by footprint, each device runs one
    batch.  Returns (ranks, device per matrix)."""
    keep = []
    nm = len(mats)
    m = np.array([int(x[3]) for x in mats], np.int64)
    n = np.array([int(x[4]) for x in mats], np.int64)
    devs = np.ascontiguousarray(devices, np.int32)
    ranks = np.zeros(nm, np.int64)
    where = np.zeros(nm, np.int32)
    check(lib().rr_batch_ranks_multi(ptr(devs), devs.size, nm, ptr(m), ptr(n),
                                     _pointer_arrays(keep, [x[0] for x in mats], np.int64),
                                     _pointer_arrays(keep, [x[1] for x in mats], np.int32),
                                     _pointer_arrays(keep, [x[2] for x in mats], np.uint32), int(theprime), int(num_v),
                                     _pointer_arrays(keep, row_preconds, np.uint32),
                                     _pointer_arrays(keep, col_preconds, np.uint32), _pointer_arrays(keep, vs, np.uint32),
                                     int(workers), ptr(ranks), ptr(where)))
    return ranks, where


class Fleet(Server):
    """Rank services on several GPUs (rr_fleet_*): each request is placed on
    the device whose service has the most budget left, and follows
    :class:`Server`'s path there."""

    def __init__(self, num_v: int, theprime: int = DEFAULT_PRIME, devices=(0,), lanes: int = 4, workers: int = 4,
                 max_active: int = 64, chunk_apps: int = 64, hbm_budget: int = 0):
        from ._lib import ServerConfig

        cfg = ServerConfig(int(num_v), int(theprime), int(lanes), int(workers), int(max_active), int(chunk_apps),
                           int(hbm_budget))
        devs = np.ascontiguousarray(devices, np.int32)
        h = C.c_void_p()
        check(lib().rr_fleet_create(ptr(devs), devs.size, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.b = int(num_v)
        _track(self, 0)

    def submit(self, rowptr, col, val, m: int, n: int, row_precond, col_precond, v) -> int:
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.uint32)
        rp = np.ascontiguousarray(row_precond, np.uint32)
        cp = np.ascontiguousarray(col_precond, np.uint32)
        v = np.ascontiguousarray(v, np.uint32)
        if rp.size != m or cp.size != n or v.shape != (self.b, n):
            raise ValueError("preconditioner or block shapes do not match the matrix")
        rid = C.c_uint64()
        check(lib().rr_fleet_submit(self.handle, m, n, ptr(rowptr), ptr(col), ptr(val), ptr(rp), ptr(cp), ptr(v),
                                    C.byref(rid)))
        return rid.value

    def result(self, rid: int, timeout: float = -1.0):
        r, lat = C.c_int64(), C.c_double()
        check(lib().rr_fleet_wait(self.handle, rid, float(timeout), C.byref(r), C.byref(lat)))
        return r.value, lat.value

    def device_of(self, rid: int) -> int:
        d = C.c_int32()
        check(lib().rr_fleet_device_of(self.handle, rid, C.byref(d)))
        return d.value

    def stats(self):
        a, b = C.c_int64(), C.c_int64()
        p50, p99, rps = C.c_double(), C.c_double(), C.c_double()
        check(lib().rr_fleet_stats(self.handle, C.byref(a), C.byref(b), C.byref(p50), C.byref(p99), C.byref(rps)))
        return {"submitted": a.value, "completed": b.value, "p50_ms": p50.value, "p99_ms": p99.value,
                "ranks_per_s": rps.value}

    def close(self):
        if getattr(self, "handle", None):
            lib().rr_fleet_destroy(self.handle)
            self.handle = None


def save_wdm_file_sym(path: str, n_rows: int, n_cols: int, theprime: int, row_precond, col_precond, v, curv, seq):
    """src/wdm_files.rs:126-210."""
    v = np.ascontiguousarray(v, np.uint32)
    curv = np.ascontiguousarray(curv, np.uint32)
    seq = np.ascontiguousarray(seq, np.uint32)
    check(lib().rr_wdm_save(path.encode(), n_rows, n_cols, theprime, v.shape[0],
                            ptr(np.ascontiguousarray(row_precond, np.uint32)),
                            ptr(np.ascontiguousarray(col_precond, np.uint32)), ptr(v), ptr(curv), ptr(seq),
                            seq.shape[1], seq.shape[1]))


def load_wdm_file_sym(path: str):
    """src/wdm_files.rs:22-123 -> (p, m, n, num_v, row_precond, col_precond, v, curv, seq)."""
    L = lib()
    m, n, nlen = C.c_int64(), C.c_int64(), C.c_int64()
    p, b = C.c_uint32(), C.c_int32()
    check(L.rr_wdm_load(path.encode(), C.byref(m), C.byref(n), C.byref(p), C.byref(b), C.byref(nlen), None, None,
                        None, None, None, 0))
    rp = np.zeros(m.value, np.uint32)
    cp = np.zeros(n.value, np.uint32)
    v = np.zeros((b.value, n.value), np.uint32)
    cv = np.zeros((b.value, n.value), np.uint32)
    seq = np.zeros((b.value * (b.value + 1) // 2, max(nlen.value, 1)), np.uint32)
    check(L.rr_wdm_load(path.encode(), C.byref(m), C.byref(n), C.byref(p), C.byref(b), C.byref(nlen), ptr(rp),
                        ptr(cp), ptr(v), ptr(cv), ptr(seq), seq.shape[1]))
    return p.value, m.value, n.value, b.value, rp, cp, v, cv, seq[:, : nlen.value]
