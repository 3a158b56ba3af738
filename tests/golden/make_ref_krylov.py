"""Golden Krylov sequences made by the reference's own GPU Krylov program.

The reference's CUDA Krylov loop (cuda_test/cuvseq_int.cu of wilthoma/rust_rank)
is built unchanged for sm_100a by

    make -C oracle REF_DIR=<checkout>/cuda_test       (-> oracle/_ref/cuvseq_int)

and run on a GPU by this script.  The random preconditioners and starting
block are injected the way the reference resumes a run: a .wdm checkpoint
with sequence length 0 (cuvseq_int.cu:477-560 loads row_precond, col_precond,
v and curv from it, then computes S_0 = curv^T curv and two sequence terms per
application of B = D_c A^T D_r A D_c, cuvseq_int.cu:817-955).  The program
writes the sequence back into the same .wdm file (save_wdm_file_sym, upper
triangle in the pair order i <= j), which is read here and stored as

    tests/golden/ref_krylov_matrix_txt.npz
        for each case "b<b>": row_precond, col_precond, V, seq [b(b+1)/2][len],
        curv [b][n] (the block after the last application), p, len

The matrix is the reference's fixture cuda_test/matrix.txt, taken from
tests/golden/matrix_txt.npz (written in the SMS text format the program reads).
The reference's int32 arithmetic restricts it to small primes: p = 3323.

    python tests/golden/make_ref_krylov.py --out tests/golden/ref_krylov_matrix_txt.npz
"""
from __future__ import annotations

import argparse
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
BIN = os.path.join(ROOT, "oracle", "_ref", "cuvseq_int")
P = 3323
# (b, sequence length N, seed)
CASES = [(8, 41, 801), (3, 61, 302), (1, 33, 103)]


def write_sms(path, rowptr, col, sval, m, n):
    with open(path, "w") as f:
        f.write(f"{m} {n} M\n")
        for r in range(m):
            for k in range(rowptr[r], rowptr[r + 1]):
                f.write(f"{r + 1} {int(col[k]) + 1} {int(sval[k])}\n")
        f.write("0 0 0\n")


def write_wdm_start(path, m, n, p, rp, cp, V):
    """A .wdm checkpoint with an empty sequence: header 'm n p 0 b', then
    row_precond, col_precond, b lines of v and b lines of curv (= v)."""
    b = V.shape[0]
    with open(path, "w") as f:
        f.write(f"{m} {n} {p} 0 {b}\n")
        f.write(" ".join(map(str, rp.tolist())) + "\n")
        f.write(" ".join(map(str, cp.tolist())) + "\n")
        for _ in range(2):
            for i in range(b):
                f.write(" ".join(map(str, V[i].tolist())) + "\n")
        for _ in range(b * (b + 1) // 2):
            f.write("\n")


def read_wdm(path):
    with open(path) as f:
        tok = f.read().split()
    m, n, p, nlen, b = (int(x) for x in tok[:5])
    pos = 5

    def take(k):
        nonlocal pos
        a = np.array(tok[pos:pos + k], dtype=np.int64)
        pos += k
        return a

    rp = take(m)
    cp = take(n)
    v = take(b * n).reshape(b, n)
    curv = take(b * n).reshape(b, n)
    seq = take(b * (b + 1) // 2 * nlen).reshape(b * (b + 1) // 2, nlen)
    assert pos == len(tok), "trailing data in the .wdm file"
    return m, n, p, nlen, b, rp, cp, v, curv, seq


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "ref_krylov_matrix_txt.npz"))
    args = ap.parse_args()
    if not os.path.exists(BIN):
        raise SystemExit("oracle/_ref/cuvseq_int missing: build it with make -C oracle REF_DIR=<checkout>/cuda_test")
    z = np.load(os.path.join(ROOT, "tests", "golden", "matrix_txt.npz"))
    rowptr, col, sval, m, n = z["rowptr"], z["col"], z["val"], int(z["m"]), int(z["n"])
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        sms = os.path.join(tmp, "matrix.txt")
        write_sms(sms, rowptr, col, sval, m, n)
        for b, N, seed in CASES:
            rng = np.random.default_rng(seed)
            rp = rng.integers(1, P, size=m)
            cp = rng.integers(1, P, size=n)
            V = rng.integers(0, P, size=(b, n))
            wdm = os.path.join(tmp, f"b{b}.wdm")
            write_wdm_start(wdm, m, n, P, rp, cp, V)
            r = subprocess.run([BIN, sms, "-f", wdm, "-N", str(N), "-p", str(P), "-v", str(b)],
                               capture_output=True, text=True, timeout=300)
            if r.returncode != 0:
                raise SystemExit(f"cuvseq_int failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
            m2, n2, p2, nlen, b2, rp2, cp2, v2, curv, seq = read_wdm(wdm)
            assert (m2, n2, p2, b2) == (m, n, P, b)
            assert np.array_equal(rp2, rp) and np.array_equal(cp2, cp) and np.array_equal(v2, V)
            key = f"b{b}"
            out[key + "_row_precond"] = rp.astype(np.uint32)
            out[key + "_col_precond"] = cp.astype(np.uint32)
            out[key + "_V"] = V.astype(np.uint32)
            out[key + "_seq"] = seq.astype(np.uint32)
            out[key + "_curv"] = curv.astype(np.uint32)
            print(f"b={b}: {nlen} terms, S_0[0] = {seq[0, 0]}, S_last[0] = {seq[0, -1]}")
    out["p"] = np.array(P)
    out["cases"] = np.array([c[0] for c in CASES])
    np.savez_compressed(args.out, **out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
