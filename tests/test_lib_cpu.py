"""Host-side checks of the CUDA library that need no GPU: it loads, exports
every entry point include/rr_rank.h declares, and its host-only entry points
(.wdm / SMS files, rank readout, prime check) behave like the reference."""
import os
import re

import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import _lib, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "rr_rank.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
        assert s in _lib.SIGNATURES, s
    assert L.rr_version().decode().startswith("rr_b200")


def test_prime_check():
    L = _lib.lib()
    assert L.rr_prime_check(2013265921) == 0
    assert L.rr_prime_check(3323) == 0
    assert L.rr_prime_check(2013265923) == 2  # divisible by 3
    assert L.rr_prime_check(2147483659) == 2  # prime but >= 2^31
    assert L.rr_prime_check(2) == 2


def test_wdm_roundtrip(tmp_path):
    p = 2013265921
    m, n, b, L = 5, 7, 3, 9
    rng = np.random.default_rng(0)
    rp = rng.integers(1, p, m).astype(np.uint32)
    cp = rng.integers(1, p, n).astype(np.uint32)
    v = rng.integers(0, p, (b, n)).astype(np.uint32)
    cv = rng.integers(0, p, (b, n)).astype(np.uint32)
    seq = rng.integers(0, p, (b * (b + 1) // 2, L)).astype(np.uint32)
    path = str(tmp_path / "x_3.wdm")
    rr.save_wdm_file_sym(path, m, n, p, rp, cp, v, cv, seq)
    first = open(path).readline().split()
    assert first == [str(m), str(n), str(p), str(L), str(b)]  # src/wdm_files.rs:144-152
    pp, mm, nn, bb, rp2, cp2, v2, cv2, seq2 = rr.load_wdm_file_sym(path)
    assert (pp, mm, nn, bb) == (p, m, n, b)
    for x, y in ((rp, rp2), (cp, cp2), (v, v2), (cv, cv2), (seq, seq2)):
        assert np.array_equal(x, y)


def test_wdm_load_errors(tmp_path):
    path = tmp_path / "bad.wdm"
    path.write_text("3 2 7 2 1\n1 2 3\n1 2\n0 1\n0\n")  # curv line too short
    with pytest.raises(rr.RRError) as e:
        rr.load_wdm_file_sym(str(path))
    assert e.value.status == 6 and "curv" in str(e.value)
    (tmp_path / "hdr.wdm").write_text("3 x 7\n")
    with pytest.raises(rr.RRError):
        rr.load_wdm_file_sym(str(tmp_path / "hdr.wdm"))
    with pytest.raises(rr.RRError):
        rr.load_wdm_file_sym(str(tmp_path / "missing.wdm"))


def test_sms_loader_matches_fixture(tmp_path, matrix_txt):
    rowptr, col, sval, m, n = matrix_txt
    lines = [f"{m} {n} M"]
    for r in range(m):
        for k in range(rowptr[r], rowptr[r + 1]):
            lines.append(f"{r + 1} {col[k] + 1} {sval[k]}")
    lines.append("0 0 0")
    path = tmp_path / "matrix.sms"
    path.write_text("% comment\n" + "\n".join(lines) + "\n")
    for p in (3323, 2013265921):
        a = rr.CsrMatrix.load_csr_matrix_from_sms(str(path), p)
        assert (a.n_rows, a.n_cols) == (m, n)
        assert np.array_equal(a.row_ptr, rowptr) and np.array_equal(a.col_indices, col)
        assert np.array_equal(a.values, (sval.astype(np.int64) % p).astype(np.uint32))
        assert a.max_nnzs() == (12, 13)
        ref = synth.load_sms(str(path), p)
        assert np.array_equal(ref[0], a.row_ptr) and np.array_equal(ref[2], a.values)


def test_rank_readout_matches_reference_golden(golden):
    z = golden("pm_basis_ref.npz")
    checked = 0
    for i in range(int(z["count"])):
        b, d, rank = (int(x) for x in z[f"c{i}_meta"])
        M, delta = z[f"c{i}_M"], z[f"c{i}_delta"]
        orc = oracle.rank_from_basis(M.astype(np.uint64), delta, 3323)
        if orc < 0:
            with pytest.raises(rr.RRError) as e:
                rr.analyze_pm_basis(M, delta, 3323)
            assert e.value.status == 7
            continue
        assert rr.analyze_pm_basis(M, delta, 3323) == rank == orc
        checked += 1
    assert checked >= 10


def test_default_sequence_length_rule():
    # src/main.rs:497-504
    assert rr.default_max_nlen(182, 168, 1) == 340
    assert rr.default_max_nlen(182, 168, 4) == 128
    assert rr.default_max_nlen(20000, 20000, 8) == 8192


def test_sms_loader_edge_cases(tmp_path):
    p = 2013265921
    # comments, blank lines, a non-positive index (skipped), negative values,
    # rows out of order (grouped by row, file order kept inside a row)
    text = "% header next\n\n3 4 M\n2 1 -1\n1 4 5\n0 2 9\n2 3 -7\n1 1 2\n3 2 1\n0 0 0\n"
    (tmp_path / "a.sms").write_text(text)
    a = rr.CsrMatrix.load_csr_matrix_from_sms(str(tmp_path / "a.sms"), p)
    assert (a.n_rows, a.n_cols) == (3, 4)
    assert a.row_ptr.tolist() == [0, 2, 4, 5]
    assert a.col_indices.tolist() == [3, 0, 0, 2, 1]
    assert a.values.tolist() == [5, 2, p - 1, p - 7, 1]
    # an entry outside the declared shape, and a file without a header line
    (tmp_path / "b.sms").write_text("2 2 M\n3 1 1\n")
    with pytest.raises(rr.RRError) as e:
        rr.CsrMatrix.load_csr_matrix_from_sms(str(tmp_path / "b.sms"), p)
    assert "outside" in str(e.value)
    (tmp_path / "c.sms").write_text("% only a comment\n")
    with pytest.raises(rr.RRError):
        rr.CsrMatrix.load_csr_matrix_from_sms(str(tmp_path / "c.sms"), p)


def test_rank_readout_rejects_bad_degrees():
    b, len_ = 2, 5
    M = np.zeros((2 * b, 2 * b, len_), np.uint32)
    with pytest.raises(rr.RRError):  # -delta beyond the basis length
        rr.analyze_pm_basis(M, np.array([-len_, 0, 0, 0], np.int64), 3323)
    with pytest.raises(rr.RRError) as e:  # degree 0 generator: no estimate
        M[0, 0, 0] = M[1, 1, 0] = 1
        rr.analyze_pm_basis(M, np.zeros(2 * b, np.int64), 3323)
    assert e.value.status == 7
