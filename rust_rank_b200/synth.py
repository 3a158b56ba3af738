"""Seeded synthetic workloads with the shapes of the block-Wiedemann benchmarks.

The reference's own matrices (graph-complex SMS files) are not distributed,
so these generators stand in for them with the sizes, sparsity and value
distributions of the five benchmark configurations:

* ``plain_single``   -- square CSR, k uniform columns per row, values +-1/+-2,
  the last ``dep_rows`` rows are seeded +-1 combinations of 3 earlier rows.
* ``zipf_large``     -- tall CSR with k distinct columns per row drawn from a
  Zipf(s) law over a random column order, values uniform in [1, p-1], plus
  duplicated rows.
* ``incidence_batch`` -- many signed-incidence style matrices (+-1 entries).

Every generator is a pure function of its seed (numpy PCG64).  Matrices are
returned as (rowptr int64, col int32, val uint32 in [0, p), m, n).
"""
from __future__ import annotations

import numpy as np

P_DEFAULT = 2013265921  # 15 * 2^27 + 1


def _csr_from_rows(cols2d: np.ndarray, vals2d: np.ndarray, m: int):
    k = cols2d.shape[1]
    order = np.argsort(cols2d, axis=1, kind="stable")
    cols = np.take_along_axis(cols2d, order, axis=1)
    vals = np.take_along_axis(vals2d, order, axis=1)
    rowptr = np.arange(0, (m + 1) * k, k, dtype=np.int64)
    return rowptr, cols.reshape(-1).astype(np.int32), vals.reshape(-1).astype(np.uint32)


def _distinct_uniform_cols(rng, m: int, n: int, k: int) -> np.ndarray:
    cols = rng.integers(0, n, size=(m, k), dtype=np.int64)
    for _ in range(64):
        s = np.sort(cols, axis=1)
        dup = np.zeros_like(cols, dtype=bool)
        dup_sorted = np.zeros_like(s, dtype=bool)
        dup_sorted[:, 1:] = s[:, 1:] == s[:, :-1]
        rows = np.nonzero(dup_sorted.any(axis=1))[0]
        if rows.size == 0:
            return cols
        # redraw whole rows that contain a repeated column
        cols[rows] = rng.integers(0, n, size=(rows.size, k), dtype=np.int64)
        del dup
    raise RuntimeError("could not draw distinct columns")


def plain_single(n: int = 20000, k: int = 6, dep_rows: int = 500, p: int = P_DEFAULT, seed: int = 43):
    """Config 1: n x n, k uniform columns per row, values +-1/+-2 mod p.

    The last ``dep_rows`` rows are +-1 combinations of 3 earlier rows (merged
    CSR rows), so rank <= n - dep_rows.
    """
    rng = np.random.default_rng(seed)
    base = n - dep_rows
    cols = _distinct_uniform_cols(rng, base, n, k)
    mags = rng.integers(1, 3, size=(base, k))
    signs = rng.integers(0, 2, size=(base, k)) * 2 - 1
    ivals = (mags * signs).astype(np.int64)
    rows_c = [c for c in cols]
    rows_v = [v for v in ivals]
    for _ in range(dep_rows):
        src = rng.choice(base, size=3, replace=False)
        coef = rng.integers(0, 2, size=3) * 2 - 1
        acc: dict[int, int] = {}
        for s, cf in zip(src, coef):
            for c, v in zip(rows_c[s], rows_v[s]):
                acc[int(c)] = acc.get(int(c), 0) + int(cf) * int(v)
        items = sorted((c, v) for c, v in acc.items() if v % p != 0)
        rows_c.append(np.array([c for c, _ in items], np.int64))
        rows_v.append(np.array([v for _, v in items], np.int64))
    rowptr = np.zeros(n + 1, np.int64)
    lens = np.array([len(r) for r in rows_c], np.int64)
    rowptr[1:] = np.cumsum(lens)
    col = np.zeros(int(rowptr[-1]), np.int32)
    val = np.zeros(int(rowptr[-1]), np.uint32)
    for r in range(n):
        c = np.asarray(rows_c[r], np.int64)
        v = np.asarray(rows_v[r], np.int64)
        o = np.argsort(c, kind="stable")
        col[rowptr[r]:rowptr[r + 1]] = c[o]
        val[rowptr[r]:rowptr[r + 1]] = (v[o] % p).astype(np.uint32)
    return rowptr, col, val, n, n


def zipf_large(m: int = 2_000_000, n: int = 1_500_000, k: int = 12, s: float = 1.1, dup_rows: int = 10_000,
               p: int = P_DEFAULT, seed: int = 44):
    """Config 2: m x n, k distinct Zipf(s) columns per row, values U[1, p-1], dup_rows duplicated rows."""
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    colmap = rng.permutation(n).astype(np.int64)

    def draw(shape):
        u = rng.random(shape)
        return colmap[np.minimum(np.searchsorted(cdf, u, side="right"), n - 1)]

    base = m - dup_rows
    cols = draw((base, k))
    for _ in range(200):
        srt = np.sort(cols, axis=1)
        bad = np.nonzero((srt[:, 1:] == srt[:, :-1]).any(axis=1))[0]
        if bad.size == 0:
            break
        # redraw only the repeated slots of the offending rows
        sub = cols[bad]
        o = np.argsort(sub, axis=1, kind="stable")
        ss = np.take_along_axis(sub, o, axis=1)
        rep = np.zeros_like(ss, dtype=bool)
        rep[:, 1:] = ss[:, 1:] == ss[:, :-1]
        fresh = draw(ss.shape)
        ss = np.where(rep, fresh, ss)
        cols[bad] = ss
    else:
        raise RuntimeError("could not draw distinct Zipf columns")
    vals = rng.integers(1, p, size=(base, k), dtype=np.int64)
    src = rng.integers(0, base, size=dup_rows)
    cols = np.concatenate([cols, cols[src]], axis=0)
    vals = np.concatenate([vals, vals[src]], axis=0)
    perm = rng.permutation(m)
    cols = cols[perm]
    vals = vals[perm]
    rowptr, col, val = _csr_from_rows(cols, vals, m)
    return rowptr, col, val, m, n


def incidence(m: int, n: int, kmin: int = 3, kmax: int = 10, deficit: int = 0, p: int = P_DEFAULT,
              seed: int = 45):
    """One signed-incidence style matrix: rows with kmin..kmax entries of value +-1.

    ``deficit`` trailing rows are +-1 combinations of 2 earlier rows.
    """
    rng = np.random.default_rng(seed)
    base = m - deficit
    lens = rng.integers(kmin, kmax + 1, size=base)
    rows_c, rows_v = [], []
    for r in range(base):
        c = rng.choice(n, size=min(int(lens[r]), n), replace=False)
        v = rng.integers(0, 2, size=c.size) * 2 - 1
        rows_c.append(c.astype(np.int64))
        rows_v.append(v.astype(np.int64))
    for _ in range(deficit):
        a, b = rng.choice(base, size=2, replace=False)
        acc: dict[int, int] = {}
        for s, cf in ((a, 1), (b, int(rng.integers(0, 2)) * 2 - 1)):
            for c, v in zip(rows_c[s], rows_v[s]):
                acc[int(c)] = acc.get(int(c), 0) + cf * int(v)
        items = sorted((c, v) for c, v in acc.items() if v % p != 0)
        rows_c.append(np.array([c for c, _ in items], np.int64))
        rows_v.append(np.array([v for _, v in items], np.int64))
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum([len(r) for r in rows_c])
    col = np.zeros(int(rowptr[-1]), np.int32)
    val = np.zeros(int(rowptr[-1]), np.uint32)
    for r in range(m):
        c = rows_c[r]
        o = np.argsort(c, kind="stable")
        col[rowptr[r]:rowptr[r + 1]] = c[o]
        val[rowptr[r]:rowptr[r + 1]] = (rows_v[r][o] % p).astype(np.uint32)
    return rowptr, col, val, m, n


def incidence_fast(m: int, n: int, kmin: int = 3, kmax: int = 10, col_deficit: int = 0, p: int = P_DEFAULT,
                   seed: int = 46):
    """Vectorised signed-incidence style matrix for large batches.

    Row r draws kmin..kmax columns uniformly (a repeated draw is dropped, so a
    row may come out one entry short) with values +-1.  Then ``col_deficit``
    columns are overwritten by copies of other columns, so the rank is at most
    n - col_deficit (the matrices are tall, so dependent rows would not lower
    the rank).
    """
    rng = np.random.default_rng(seed)
    lens = rng.integers(kmin, kmax + 1, size=m)
    cand = np.sort(rng.integers(0, n, size=(m, kmax), dtype=np.int64), axis=1)
    keep = np.arange(kmax)[None, :] < lens[:, None]
    keep[:, 1:] &= cand[:, 1:] != cand[:, :-1]
    rows = np.broadcast_to(np.arange(m, dtype=np.int64)[:, None], cand.shape)[keep]
    cols = cand[keep]
    vals = rng.integers(0, 2, size=cols.size, dtype=np.int64) * 2 - 1
    if col_deficit > 0:
        pick = rng.permutation(n)[: 2 * col_deficit]
        src, dst = pick[:col_deficit], pick[col_deficit:]
        drop = np.isin(cols, dst)
        rows, cols, vals = rows[~drop], cols[~drop], vals[~drop]
        where = np.full(n, -1, np.int64)
        where[src] = dst
        sel = where[cols] >= 0
        rows = np.concatenate([rows, rows[sel]])
        vals = np.concatenate([vals, vals[sel]])
        cols = np.concatenate([cols, where[cols[sel]]])
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum(np.bincount(rows, minlength=m))
    return rowptr, cols.astype(np.int32), (vals % p).astype(np.uint32), m, n


def graph_complex_batch(nmat: int = 256, rmin: int = 1000, rmax: int = 200_000, kmin: int = 3, kmax: int = 10,
                        deficit_every: int = 8, p: int = P_DEFAULT, seed: int = 47):
    """Config 3: ``nmat`` incidence-style matrices, rows log-uniform in
    [rmin, rmax], columns = rows * U(0.6, 1.0); every ``deficit_every``-th
    matrix gets a planted column deficit of about 1% of its columns."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(rmin), np.log(rmax), size=nmat)).astype(np.int64)
    frac = rng.uniform(0.6, 1.0, size=nmat)
    mats = []
    for i in range(nmat):
        m = int(rows[i])
        n = max(1, int(m * frac[i]))
        dfc = (n // 100 + 1) if deficit_every and i % deficit_every == 0 else 0
        mats.append(incidence_fast(m, n, kmin, kmax, dfc, p, seed * 1000 + i))
    return mats


def random_vectors(b: int, n: int, p: int, seed: int, nonzero: bool = False) -> np.ndarray:
    """b x n uniform in [0, p) (or [1, p) with nonzero), like src/matrices.rs:484-497."""
    rng = np.random.default_rng(seed)
    lo = 1 if nonzero else 0
    return rng.integers(lo, p, size=(b, n), dtype=np.int64).astype(np.uint32)


def preconditioners(m: int, n: int, p: int, seed: int):
    """Row and column diagonal preconditioners, uniform in [1, p-1] (src/main.rs:463-465)."""
    rng = np.random.default_rng(seed)
    return (rng.integers(1, p, size=m, dtype=np.int64).astype(np.uint32),
            rng.integers(1, p, size=n, dtype=np.int64).astype(np.uint32))


def load_sms(path: str, p: int):
    """Parse an SMS file like src/matrices.rs:662-732 (1-based triplets, value mod p)."""
    rows, cols, vals = [], [], []
    m = n = 0
    have_header = False
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("%"):
                continue
            parts = line.split()
            if len(parts) == 3 and not have_header:
                m, n = int(parts[0]), int(parts[1])
                have_header = True
                continue
            if len(parts) != 3:
                continue
            r, c, v = int(parts[0]), int(parts[1]), int(parts[2])
            if r <= 0 or c <= 0:
                continue
            rows.append(r - 1)
            cols.append(c - 1)
            vals.append(v % p)
    rows = np.asarray(rows, np.int64)
    counts = np.bincount(rows, minlength=m) if rows.size else np.zeros(m, np.int64)
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum(counts)
    order = np.argsort(rows, kind="stable")
    col = np.asarray(cols, np.int64)[order].astype(np.int32)
    val = np.asarray(vals, np.int64)[order].astype(np.uint32)
    return rowptr, col, val, m, n
