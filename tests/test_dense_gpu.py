"""GPU dense complex LU / solves / GEMM (libbem200) against scipy LAPACK."""
import ctypes

import numpy as np
import pytest
import scipy.linalg as sla

from mnpbem_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _rand(n, m, seed, dtype=np.complex128):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(dtype)


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def getrf(A, engine=0):
    import torch
    n = A.shape[0]
    code = nat.C128 if A.dtype == torch.complex128 else nat.C64
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_getrf", code, engine, n, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info), None,
             0, nat.stream_ptr())
    return rowmap, ipiv, info


def getrs(LU, rowmap, B):
    import torch
    n, nrhs = B.shape
    code = nat.C128 if B.dtype == torch.complex128 else nat.C64
    scr = torch.empty(int(nat.lib().bem200_getrs_workspace_size(code, n, nrhs)), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_getrs", code, 0, n, nrhs, nat.ptr(LU), n, nat.ptr(rowmap), nat.ptr(B), nrhs, None, 0,
             nat.ptr(scr), nat.ptr(status), nat.stream_ptr())
    assert int(status.item()) == 0


@pytest.mark.parametrize("n", [33, 300, 1100])
def test_getrf_c128_matches_lapack(cuda, n):
    A = _rand(n, n, n)
    At = _t(A)
    rowmap, ipiv, info = getrf(At)
    lu, piv = sla.lu_factor(A)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    # storage rows are not moved: logical row i lives in storage row rowmap[i]
    got = At.cpu().numpy()[rowmap.cpu().numpy()]
    err = np.max(np.abs(got - lu)) / np.max(np.abs(lu))
    assert err < 1e-11


@pytest.mark.parametrize("n,nrhs", [(300, 1), (700, 5), (1000, 16), (1100, 1100), (77, 3)])
def test_getrs_c128(cuda, n, nrhs):
    A = _rand(n, n, 7)
    B = _rand(n, nrhs, 8)
    At, Bt = _t(A), _t(B)
    rowmap, _, _ = getrf(At)
    getrs(At, rowmap, Bt)
    X = np.linalg.solve(A, B)
    assert np.max(np.abs(Bt.cpu().numpy() - X)) / np.max(np.abs(X)) < 1e-10


def test_getrf_c64(cuda):
    n = 900
    A = _rand(n, n, 3)
    At = _t(A.astype(np.complex64))
    rowmap, ipiv, info = getrf(At)
    B = _rand(n, 4, 4)
    Bt = _t(B.astype(np.complex64))
    getrs(At, rowmap, Bt)
    X = np.linalg.solve(A, B)
    assert np.max(np.abs(Bt.cpu().numpy() - X)) / np.max(np.abs(X)) < 1e-3


@pytest.mark.parametrize("dt,tol", [(np.complex128, 1e-13), (np.complex64, 1e-5)])
def test_gemm(cuda, dt, tol):
    m, n, k = 257, 190, 333
    A, B, C = _rand(m, k, 1, dt), _rand(k, n, 2, dt), _rand(m, n, 3, dt)
    At, Bt, Ct = _t(A), _t(B), _t(C)
    alpha = (ctypes.c_double * 2)(0.5, -1.0)
    beta = (ctypes.c_double * 2)(1.0, 0.25)
    code = nat.C128 if dt == np.complex128 else nat.C64
    nat.call("bem200_gemm", code, 0, m, n, k, alpha, nat.ptr(At), k, nat.ptr(Bt), n, beta, nat.ptr(Ct), n, None, 0,
             nat.stream_ptr())
    ref = (0.5 - 1j) * (A.astype(np.complex128) @ B) + (1 + 0.25j) * C
    assert np.max(np.abs(Ct.cpu().numpy() - ref)) / np.max(np.abs(ref)) < tol


def test_singular_pivot_reported(cuda):
    A = _rand(64, 64, 5)
    A[:, 10] = 0
    At = _t(A)
    _, _, info = getrf(At)
    assert int(info.item()) == 11


@pytest.mark.parametrize("dt,tol", [(np.complex128, 1e-13), (np.complex64, 1e-5)])
@pytest.mark.parametrize("n", [1, 4, 8, 12, 16])
def test_gemm_skinny(cuda, dt, tol, n):
    """Matrix times few vectors (n <= 16, k >= 256): the bandwidth-bound skinny kernel."""
    m, k = 1000, 700
    A, B, C = _rand(m, k, 11, dt), _rand(k, n, 12, dt), _rand(m, n, 13, dt)
    At, Bt, Ct = _t(A), _t(B), _t(C)
    alpha = (ctypes.c_double * 2)(1.5, 0.5)
    beta = (ctypes.c_double * 2)(-0.5, 2.0)
    code = nat.C128 if dt == np.complex128 else nat.C64
    nat.call("bem200_gemm", code, 0, m, n, k, alpha, nat.ptr(At), k, nat.ptr(Bt), n, beta, nat.ptr(Ct), n, None, 0,
             nat.stream_ptr())
    ref = (1.5 + 0.5j) * (A.astype(np.complex128) @ B) + (-0.5 + 2j) * C
    assert np.max(np.abs(Ct.cpu().numpy() - ref)) / np.max(np.abs(ref)) < tol


def _getrf_ws(A, engine, flags=0):
    """getrf with its full workspace: the look-ahead (two-stream) schedule."""
    import torch
    n = A.shape[0]
    code = nat.C128 if A.dtype == torch.complex128 else nat.C64
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = int(nat.lib().bem200_getrf_workspace_size(code, engine, n))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    nat.call("bem200_getrf_ex", code, engine, n, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
             nat.ptr(ws), wsb, flags, 0, nat.stream_ptr())
    return rowmap, ipiv, info


@pytest.mark.parametrize("n", [300, 1100, 1537])
def test_getrf_lookahead_c128_matches_lapack(cuda, n):
    A = _rand(n, n, 40 + n)
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, 0)
    lu, piv = sla.lu_factor(A)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    got = At.cpu().numpy()[rowmap.cpu().numpy()]
    assert np.max(np.abs(got - lu)) / np.max(np.abs(lu)) < 1e-11


def test_getrf_lookahead_c64_tensor_cores(cuda):
    """complex64 look-ahead LU on the bf16x3 tensor-core engine, on a
    well-conditioned matrix (cond ~ 3, as the bf16x3 products carry ~2^-16
    relative error): the solve error matches the single-stream schedule's."""
    n = 1500
    A = (_rand(n, n, 77) / np.sqrt(n) + 3 * np.eye(n)).astype(np.complex64)
    B = _rand(n, 3, 78)
    X = np.linalg.solve(A.astype(np.complex128), B)
    errs = []
    for lookahead in (True, False):
        At = _t(A)
        if lookahead:
            rowmap, ipiv, info = _getrf_ws(At, 1)
        else:
            import torch
            rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
            ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
            info = torch.zeros(1, dtype=torch.int32, device="cuda")
            wsb = int(nat.lib().bem200_gemm_workspace_size(1, n, n, n))  # too small for look-ahead
            ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
            nat.call("bem200_getrf", nat.C64, 1, n, nat.ptr(At), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
                     nat.ptr(ws), wsb, nat.stream_ptr())
        assert int(info.item()) == 0
        Bt = _t(B.astype(np.complex64))
        getrs(At, rowmap, Bt)
        errs.append(np.max(np.abs(Bt.cpu().numpy() - X)) / np.max(np.abs(X)))
    assert errs[0] < 2e-4 and errs[0] < 3 * errs[1] + 1e-6, errs


def test_getrf_lookahead_tall_panel_c128(cuda):
    """n = 6500 > 6144 rows: the first panels are factored by the grid-wide
    (cooperative) panel kernel; pivots and factors still match LAPACK."""
    n = 6500
    A = _rand(n, n, 2024)
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, 0)
    lu, piv = sla.lu_factor(A)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    got = At.cpu().numpy()[rowmap.cpu().numpy()]
    assert np.max(np.abs(got - lu)) / np.max(np.abs(lu)) < 1e-10


@pytest.mark.parametrize("n", [700, 3000, 5768])
def test_getrf_c64_tournament_pivoting(cuda, n):
    """BEM200_GETRF_TOURNAMENT_PIVOTING: complex64 panels of more than 512
    rows pick their pivots by tournament (one cluster exchange per panel).
    The factors solve as accurately as the default partial-pivoting ones:
    backward error of a solve within a small factor of theirs and at the
    complex64 rounding level (~2e-5 at n = 3000 for both)."""
    import torch
    A = _rand(n, n, 900 + n).astype(np.complex64)
    B = _rand(n, 2, 901 + n).astype(np.complex64)
    A64 = A.astype(np.complex128)
    berr = []
    for flags in (2, 0):
        At = _t(A)
        rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
        ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        wsb = int(nat.lib().bem200_getrf_workspace_size(nat.C64, 1, n))
        ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
        nat.call("bem200_getrf_ex", nat.C64, 1, n, nat.ptr(At), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
                 nat.ptr(ws), wsb, flags, 0, nat.stream_ptr())
        assert int(info.item()) == 0
        perm = rowmap.cpu().numpy()
        assert sorted(perm.tolist()) == list(range(n))      # a permutation
        Bt = _t(B)
        getrs(At, rowmap, Bt)
        X = Bt.cpu().numpy().astype(np.complex128)
        r = A64 @ X - B
        berr.append(np.max(np.abs(r)) / (np.max(np.sum(np.abs(A64), axis=1)) * np.max(np.abs(X))))
    assert berr[0] < 1e-4 and berr[0] < 10 * berr[1] + 1e-7, berr


@pytest.mark.parametrize("flags", [0, 2], ids=["async_panel", "tournament"])
@pytest.mark.parametrize("zcol", [10, 700])
def test_getrf_c64_zero_column(cuda, flags, zcol):
    """A zero column inside a tall complex64 panel (the asynchronous push
    panel, or a tournament panel) is reported as a zero pivot, also in a
    later panel of the look-ahead schedule."""
    n = 1200
    A = (_rand(n, n, 41) + 3 * np.eye(n)).astype(np.complex64)
    A[:, zcol] = 0
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, 1, flags=flags)
    assert int(info.item()) == zcol + 1


def test_getrf_c64_pivots_match_lapack(cuda):
    """complex64 partial pivoting (asynchronous push panels, CUDA-core
    updates) picks LAPACK cgetrf's pivots on a random 600 x 600 matrix, with
    factors equal to cgetrf's to complex64 rounding.  (On larger random
    matrices the two diverge at the first near-tie that rounding decides.)"""
    n = 600
    A = _rand(n, n, 500 + n).astype(np.complex64)
    lu, piv = sla.lu_factor(A)
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, 0)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    got = At.cpu().numpy()[rowmap.cpu().numpy()]
    assert np.max(np.abs(got - lu)) / np.max(np.abs(lu)) < 1e-4


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("n", [2000, 5768])
def test_getrf_c64_partial_pivoting_factors(cuda, n, engine):
    """complex64 look-ahead LU with asynchronous push panels: rowmap is a
    permutation consistent with ipiv, every multiplier is bounded as partial
    pivoting on |re| + |im| implies (|l| <= sqrt 2), and P A = L U holds to
    complex64 rounding (CUDA-core and bf16x3 tensor-core updates)."""
    A = _rand(n, n, 700 + n).astype(np.complex64)
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, engine)
    assert int(info.item()) == 0
    perm = rowmap.cpu().numpy()
    assert sorted(perm.tolist()) == list(range(n))
    order = np.arange(n)
    for k, q in enumerate(ipiv.cpu().numpy()):       # LAPACK swaps replayed
        order[[k, q]] = order[[q, k]]
    np.testing.assert_array_equal(order, perm)
    F = At.cpu().numpy()[perm].astype(np.complex128)
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    assert np.max(np.abs(L)) <= np.sqrt(2) * (1 + 1e-5)
    r = np.max(np.abs(A[perm].astype(np.complex128) - L @ U)) / np.max(np.abs(A))
    assert r < (5e-3 if engine else 1e-4), r  # bf16x3 products: ~2^-16 each


def _dominant(n, seed, dt):
    """A random matrix with a column-dominant diagonal: partial pivoting makes no row exchange."""
    return (_rand(n, n, seed) + 4.0 * np.sqrt(n) * np.eye(n)).astype(dt)


@pytest.mark.parametrize("n", [100, 1000, 2000])
def test_getrf_diagonal_pivots_c128_equal_lapack(cuda, n):
    """BEM200_GETRF_DIAGONAL_PIVOTS (no pivot search, blocked, checked): on a
    matrix whose partial-pivoting LU exchanges no rows, LAPACK's pivots
    (ipiv[k] = k) and its factors to FP64 rounding; block edges at n = 1000
    (not a multiple of the 64-column blocks)."""
    A = _dominant(n, 60 + n, np.complex128)
    lu, piv = sla.lu_factor(A)
    assert np.array_equal(piv, np.arange(n))
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, 0, flags=4)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    np.testing.assert_array_equal(rowmap.cpu().numpy(), np.arange(n))
    assert np.max(np.abs(At.cpu().numpy() - lu)) / np.max(np.abs(lu)) < 1e-12


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("n", [300, 1000, 5768])
def test_getrf_diagonal_pivots_c64_equal_partial(cuda, n, engine):
    """complex64 checked diagonal pivots (128-column blocks, tensor-core or
    CUDA-core trailing updates) against the partial-pivoting LU of the same
    matrix (which exchanges no rows): same pivots, factors equal to complex64
    rounding, and a solve as accurate."""
    A = _dominant(n, 80 + n, np.complex64)
    ref = _t(A)
    rmap, rpiv, rinfo = _getrf_ws(ref, engine)
    assert int(rinfo.item()) == 0 and np.array_equal(rpiv.cpu().numpy(), np.arange(n))
    At = _t(A)
    rowmap, ipiv, info = _getrf_ws(At, engine, flags=4)
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), np.arange(n))
    F, R = At.cpu().numpy(), ref.cpu().numpy()[rmap.cpu().numpy()]
    assert np.max(np.abs(F - R)) / np.max(np.abs(R)) < (2e-4 if engine else 2e-5)
    B = _rand(n, 2, 81 + n).astype(np.complex64)
    Bt = _t(B)
    getrs(At, rowmap, Bt)
    X = np.linalg.solve(A.astype(np.complex128), B)
    assert np.max(np.abs(Bt.cpu().numpy() - X)) / np.max(np.abs(X)) < 1e-4


@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
@pytest.mark.parametrize("where,off", [(3, 40), (3, 150), (700, 150)])
def test_getrf_diagonal_pivots_report_needed_exchange(cuda, dt, where, off):
    """A column whose partial-pivoting step would exchange rows -- with a row
    of the same diagonal block, or with a row below it, in the first block or
    a later one -- makes the checked LU report -BEM200_ERR_PIVOTING."""
    n = 1000
    A = _dominant(n, 90, dt)
    A[[where, where + off]] = A[[where + off, where]]   # the diagonal of row `where` moves below it
    At = _t(A)
    _, _, info = _getrf_ws(At, 1 if dt == np.complex64 else 0, flags=4)
    assert int(info.item()) == -nat.ERR_PIVOTING


@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
def test_getrf_diagonal_pivots_zero_column(cuda, dt):
    """An all-zero column needs no exchange under partial pivoting either:
    the checked LU reports the zero pivot (info = column + 1), as LAPACK."""
    n = 500
    A = _dominant(n, 91, dt)
    A[:, 200] = 0
    At = _t(A)
    _, _, info = _getrf_ws(At, 0, flags=4)
    assert int(info.item()) == 201


def _inverse_nopiv(A, engine, tol=1e-2):
    import torch
    n = A.shape[0]
    code = nat.C128 if A.dtype == torch.complex128 else nat.C64
    L = nat.lib()
    scr = torch.empty(int(L.bem200_inverse_nopiv_workspace_size(code, n)), dtype=torch.uint8, device="cuda")
    wsb = int(L.bem200_gemm_workspace_size(engine, n, n, n // 2 + 64)) if engine else 0
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("bem200_inverse_nopiv", code, engine, n, nat.ptr(A), n, nat.ptr(ws), wsb, nat.ptr(scr), tol,
             nat.ptr(info), nat.stream_ptr())
    return int(info.item())


@pytest.mark.parametrize("dt,engine,tol", [(np.complex128, 0, 1e-12), (np.complex64, 0, 2e-5),
                                           (np.complex64, 1, 2e-3)], ids=["c128", "c64-simt", "c64-bf16x3"])
@pytest.mark.parametrize("n", [100, 700, 1500])
def test_inverse_nopiv(cuda, dt, engine, tol, n):
    """bem200_inverse_nopiv (block Schur complement, Gauss-Jordan leaves, no
    pivoting) on a matrix whose partial-pivoting LU exchanges no rows: the
    inverse to the dtype's (and GEMM engine's) rounding, info = 0."""
    A = _dominant(n, 300 + n, dt)
    At = _t(A)
    assert _inverse_nopiv(At, engine) == 0
    X = At.cpu().numpy().astype(np.complex128)
    r = np.max(np.abs(X @ A.astype(np.complex128) - np.eye(n)))
    assert r < tol, r


@pytest.mark.parametrize("engine", [0, 1], ids=["simt", "bf16x3"])
def test_inverse_nopiv_graph_replay(cuda, engine):
    """The inverse's launches are recorded once per argument set and replayed
    from a CUDA graph: a repeated call on the same buffers gives the same bits
    and counts the same kernels; a replay on a side stream and the direct
    launches inside a caller's own stream capture give the same bits too."""
    import torch
    n = 700
    A0 = _t(_dominant(n, 900, np.complex64))
    A = A0.clone()
    L = nat.lib()
    scr = torch.empty(int(L.bem200_inverse_nopiv_workspace_size(nat.C64, n)), dtype=torch.uint8, device="cuda")
    wsb = int(L.bem200_gemm_workspace_size(engine, n, n, n // 2 + 64)) if engine else 0
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")

    def run(stream=None):
        A.copy_(A0)
        nat.call("bem200_inverse_nopiv", nat.C64, engine, n, nat.ptr(A), n, nat.ptr(ws), wsb, nat.ptr(scr), 1e-2,
                 nat.ptr(info), nat.stream_ptr(stream))

    c0 = int(L.bem200_launch_count())
    run()
    torch.cuda.synchronize()
    c1 = int(L.bem200_launch_count())
    X1 = A.clone()
    run()
    torch.cuda.synchronize()
    c2 = int(L.bem200_launch_count())
    assert torch.equal(A, X1)
    assert c2 - c1 == c1 - c0 > 10
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        run(side)
    side.synchronize()
    assert torch.equal(A, X1)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        run()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(A, X1)
    assert int(info.item()) == 0
    r = np.max(np.abs(X1.cpu().numpy().astype(np.complex128) @ A0.cpu().numpy().astype(np.complex128) - np.eye(n)))
    assert r < 2e-3, r
    del g


@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
def test_inverse_nopiv_reports_needed_exchange(cuda, dt):
    """A matrix whose elimination needs row exchanges (a plain random one,
    and a dominant one with two rows of a leaf swapped) gets info = 1."""
    n = 300
    A = _rand(n, n, 301).astype(dt)
    assert _inverse_nopiv(_t(A), 0) == 1
    B = _dominant(n, 302, dt)
    B[[5, 40]] = B[[40, 5]]
    assert _inverse_nopiv(_t(B), 0) == 1
