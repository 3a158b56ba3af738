"""The allocation-free PM-basis entry point (rr_pm_basis_short_noalloc).

Some callers cannot allocate device memory at the moment they need a short
generator: hosts whose device memory is owned by their own pool allocator, or
loops that cannot afford cudaMalloc's implicit synchronisation.  This entry
point serves them from a fixed scratch array inside the library; its output
must equal the regular entry point's (rr_pm_basis) and the oracle's exactly,
including on back-to-back calls that share the scratch array, and must not
carry the failure marker (every delta entry INT64_MIN).

Collected last on purpose (file name) so that a stop-at-first-failure run has
already run every other test when this one runs.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import rust_rank_b200 as rr
from rust_rank_b200 import _lib

pytestmark = pytest.mark.gpu

P = 2013265921


def noalloc_pm_basis(seq, b, d, p):
    """Call the C ABI with caller-owned device buffers (the test allocates them, not the library)."""
    import torch

    seq = np.ascontiguousarray(seq, np.uint32)
    nlen = seq.shape[1]
    dd = 1 << (d - 1).bit_length()
    d_seq = torch.from_numpy(seq.view(np.int32)).cuda()
    d_M = torch.full((2 * b, 2 * b, dd + 1), -1, dtype=torch.int32, device="cuda")
    d_delta = torch.full((2 * b,), 7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    _lib.check(_lib.lib().rr_pm_basis_short_noalloc(C.c_void_p(d_seq.data_ptr()), nlen, b, nlen, d, p,
                                                      C.c_void_p(d_M.data_ptr()), C.c_void_p(d_delta.data_ptr()),
                                                      C.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return d_M.cpu().numpy().view(np.uint32), d_delta.cpu().numpy()


@pytest.mark.parametrize("b,d,p", [(1, 32, P), (2, 8, P), (8, 32, P), (16, 32, P), (16, 5, P), (4, 16, 3323)])
def test_matches_regular_entry_point_on_two_calls(b, d, p):
    rng = np.random.default_rng(1000 * b + d)
    dd = 1 << (d - 1).bit_length()
    for call in range(2):
        seq = rng.integers(0, p, size=(b * (b + 1) // 2, dd + 1 + call)).astype(np.uint32)
        M_ref, delta_ref = rr.PM_Basis(seq, d, p)
        M, delta = noalloc_pm_basis(seq, b, d, p)
        assert not np.all(delta == np.iinfo(np.int64).min), f"call {call}: device-side failure marker"
        assert np.array_equal(M, M_ref), f"call {call}"
        assert np.array_equal(delta, delta_ref), f"call {call}"
        M_orc, delta_orc = oracle.pm_basis(seq, b, d, p)
        assert np.array_equal(M, M_orc.astype(np.uint32)), f"call {call}"
        assert np.array_equal(delta, delta_orc), f"call {call}"


def test_rejects_sizes_beyond_the_limit():
    seq = np.zeros((17 * 18 // 2, 40), np.uint32)
    with pytest.raises(rr.RRError) as e:
        noalloc_pm_basis(seq, 17, 8, P)
    assert e.value.status == 1 and "limit" in str(e.value)
    seq = np.zeros((3, 70), np.uint32)
    with pytest.raises(rr.RRError) as e:
        noalloc_pm_basis(seq, 2, 33, P)
    assert e.value.status == 1 and "limit" in str(e.value)


def test_captured_in_a_cuda_graph():
    """The stated use inside stream capture: one call before capture (it looks
    up the scratch array and sets the kernel attribute), one call captured
    into a CUDA graph on a side stream, the graph replayed on new sequences:
    each replay equals the regular entry point."""
    import torch

    b, d, p = 8, 32, P
    np_, nlen = b * (b + 1) // 2, d + 1
    rng = np.random.default_rng(77)
    d_seq = torch.zeros((np_, nlen), dtype=torch.int32, device="cuda")
    d_M = torch.zeros((2 * b, 2 * b, d + 1), dtype=torch.int32, device="cuda")
    d_delta = torch.zeros((2 * b,), dtype=torch.int64, device="cuda")

    def call(stream):
        _lib.check(_lib.lib().rr_pm_basis_short_noalloc(C.c_void_p(d_seq.data_ptr()), nlen, b, nlen, d, p,
                                                          C.c_void_p(d_M.data_ptr()), C.c_void_p(d_delta.data_ptr()),
                                                          C.c_void_p(stream.cuda_stream)))

    side = torch.cuda.Stream()
    d_seq.copy_(torch.from_numpy(rng.integers(0, p, size=(np_, nlen)).astype(np.uint32).view(np.int32)))
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        call(side)  # first call: outside capture
    side.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        call(torch.cuda.current_stream())
    for rep in range(2):
        seq = rng.integers(0, p, size=(np_, nlen)).astype(np.uint32)
        d_seq.copy_(torch.from_numpy(seq.view(np.int32)))
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        M = d_M.cpu().numpy().view(np.uint32)
        delta = d_delta.cpu().numpy()
        M_ref, delta_ref = rr.PM_Basis(seq, d, p)
        assert np.array_equal(M, M_ref), f"replay {rep}"
        assert np.array_equal(delta, delta_ref), f"replay {rep}"
    del graph
