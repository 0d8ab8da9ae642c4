"""bem200_getrs_noalloc: the triangular solve for callers that cannot allocate
device memory (a host program linking only libbem200 with no device
allocator of its own, or a caller whose device memory belongs to another
runtime's pool and that must not call cudaMalloc / cudaFree, which
synchronise the whole device).

The variant takes its scratch from a fixed buffer inside the library, so its
answers must equal those of bem200_getrs with caller-provided scratch, on
two calls in a row (the second call sees the first call's leftovers in the
shared buffer).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mnpbem_b200 import _native as nat


def _rand(n, m, seed, dtype=np.complex128):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(dtype)


def _factor(A):
    import torch
    n = A.shape[0]
    code = nat.C128 if A.dtype == torch.complex128 else nat.C64
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_getrf", code, 0, n, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info), None, 0,
             nat.stream_ptr())
    assert int(info.item()) == 0
    return rowmap


def _getrs(code, LU, rowmap, B):
    """The existing entry point with caller-allocated scratch."""
    import torch
    n, nrhs = B.shape
    scr = torch.empty(int(nat.lib().bem200_getrs_workspace_size(code, n, nrhs)), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_getrs", code, 0, n, nrhs, nat.ptr(LU), n, nat.ptr(rowmap), nat.ptr(B), nrhs, None, 0,
             nat.ptr(scr), nat.ptr(status), nat.stream_ptr())
    assert int(status.item()) == 0


def _getrs_noalloc(code, LU, rowmap, B, status):
    n, nrhs = B.shape
    nat.call("bem200_getrs_noalloc", code, n, nrhs, nat.ptr(LU), n, nat.ptr(rowmap), nat.ptr(B), nrhs,
             nat.ptr(status), nat.stream_ptr())


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
def test_noalloc_matches_getrs_two_calls(cuda):
    import torch
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    # call 1: complex128, 700 unknowns, 5 right-hand sides (blocked TRSV)
    # call 2: complex128, 1100 unknowns, 24 right-hand sides (blocked TRSM),
    #         so it reuses a buffer that call 1 left dirty
    cases = [(700, 5, 11), (1100, 24, 12)]
    for n, nrhs, seed in cases:
        A = torch.as_tensor(_rand(n, n, seed), device="cuda")
        rowmap = _factor(A)
        B0 = _rand(n, nrhs, seed + 100)
        ref = torch.as_tensor(B0, device="cuda")
        got = torch.as_tensor(B0, device="cuda")
        _getrs(nat.C128, A, rowmap, ref)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _getrs_noalloc(nat.C128, A, rowmap, got, status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        if seed == cases[-1][2]:  # the buffer is set up by now: nothing may change
            assert torch.cuda.mem_get_info()[0] == free0
        g, r = got.cpu().numpy(), ref.cpu().numpy()
        assert _rel(g, r) < 1e-12, (n, nrhs, _rel(g, r))
        X = np.linalg.solve(_rand(n, n, seed), B0)
        assert _rel(g, X) < 1e-10


@pytest.mark.gpu
def test_noalloc_complex64_repeated(cuda):
    import torch
    n = 900
    A = torch.as_tensor(_rand(n, n, 3).astype(np.complex64), device="cuda")
    rowmap = _factor(A)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for seed in (4, 5):
        B0 = _rand(n, 4, seed).astype(np.complex64)
        ref = torch.as_tensor(B0, device="cuda")
        got = torch.as_tensor(B0, device="cuda")
        _getrs(nat.C64, A, rowmap, ref)
        _getrs_noalloc(nat.C64, A, rowmap, got, status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert _rel(got.cpu().numpy(), ref.cpu().numpy()) < 1e-6


def test_noalloc_rejects_sizes_above_the_buffer():
    """Scratch beyond the fixed buffer is refused before any device work."""
    L = nat.lib()
    n, nrhs = 5768, 64  # 5768 x 64 complex128 = 5.9 MB > 4 MiB
    assert L.bem200_getrs_workspace_size(nat.C128, n, nrhs) > (4 << 20)
    st = L.bem200_getrs_noalloc(nat.C128, n, nrhs, ctypes.c_void_p(16), n, ctypes.c_void_p(16),
                                ctypes.c_void_p(16), nrhs, None, None)
    assert st == 1
    msg = nat.last_error()
    assert "getrs_noalloc" in msg and "bem200_getrs" in msg
