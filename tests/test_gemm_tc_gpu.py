"""tcgen05 tensor-core complex64 GEMM (bf16x3 split, FP32 accumulate) vs numpy."""
import ctypes

import numpy as np
import pytest

from mnpbem_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _rand(n, m, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)


# (1000, 700, 900) and (300, 301, 2000) split K over 3 and 8 slab ranges (odd n: scalar partial stores)
@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (257, 190, 333), (1000, 700, 900), (640, 1300, 96),
                                   (300, 301, 2000)])
def test_gemm_bf16x3(cuda, m, n, k):
    import torch
    A, B, C = _rand(m, k, 1), _rand(k, n, 2), _rand(m, n, 3)
    At, Bt, Ct = (torch.as_tensor(x, device="cuda") for x in (A, B, C))
    ws_bytes = int(nat.lib().bem200_gemm_workspace_size(1, m, n, k))
    ws = torch.zeros(ws_bytes, dtype=torch.uint8, device="cuda")
    alpha = (ctypes.c_double * 2)(-1.0, 0.5)
    beta = (ctypes.c_double * 2)(1.0, 0.0)
    nat.call("bem200_gemm", nat.C64, 1, m, n, k, alpha, nat.ptr(At), k, nat.ptr(Bt), n, beta, nat.ptr(Ct), n,
             nat.ptr(ws), ws_bytes, nat.stream_ptr())
    torch.cuda.synchronize()
    ref = (-1 + 0.5j) * (A.astype(np.complex128) @ B.astype(np.complex128)) + C
    got = Ct.cpu().numpy()
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-4, err


def _lu_solve_err(A, B, engine):
    import torch
    n = A.shape[0]
    At = torch.as_tensor(A.astype(np.complex64), device="cuda")
    ws_bytes = int(nat.lib().bem200_gemm_workspace_size(engine, n, n, n))
    ws = torch.zeros(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_getrf", nat.C64, engine, n, nat.ptr(At), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
             nat.ptr(ws), ws_bytes, nat.stream_ptr())
    Bt = torch.as_tensor(B.astype(np.complex64), device="cuda")
    scr = torch.empty(int(nat.lib().bem200_getrs_workspace_size(nat.C64, n, B.shape[1])), dtype=torch.uint8,
                      device="cuda")
    nat.call("bem200_getrs", nat.C64, engine, n, B.shape[1], nat.ptr(At), n, nat.ptr(rowmap), nat.ptr(Bt),
             B.shape[1], nat.ptr(ws), ws_bytes, nat.ptr(scr), None, nat.stream_ptr())
    X = np.linalg.solve(A, B)
    assert int(info.item()) == 0
    return np.max(np.abs(Bt.cpu().numpy() - X)) / np.max(np.abs(X))


def test_getrf_tensor_core_engine(cuda):
    """LU with tensor-core trailing updates on a well-conditioned matrix (cond ~ 3):
    the solution error stays at the bf16x3 level (~1e-5) and within a small
    factor of the complex64 CUDA-core LU."""
    n = 1500
    A = _rand(n, n, 11).astype(np.complex128) / np.sqrt(n) + 3 * np.eye(n)
    B = _rand(n, 4, 12).astype(np.complex128)
    err_tc = _lu_solve_err(A, B, 1)
    err_simt = _lu_solve_err(A, B, 0)
    assert err_tc < 2e-4 and err_tc < 200 * max(err_simt, 1e-7), (err_tc, err_simt)
