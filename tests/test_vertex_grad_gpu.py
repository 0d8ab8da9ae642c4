"""Reverse-mode vertex gradient of the extinction (one transposed solve with
the wavelength's factors, the operator derivative contracted on the GPU).

* the transposed solve and the transposed FP64 operator satisfy the adjoint
  identities <S^T u, v> = <u, S v> and <A^T l, x> = <l, A x>;
* the gradient matches the reference solver's own central differences
  (tests/golden/shape_fd_rod.npz: the unmodified reference BEMRet at
  v +- h D, h = 1e-4 nm) and central differences of this solver on curved
  spheres, a dimer and a flat ellipsoid.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden
from meshes import dimer, refinement_of, shape_particle, sphere

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _bem(cp, enei, precision):
    from mnpbem_b200 import BEMRet
    bem = BEMRet(cp, precision=precision)
    bem.init(enei)
    return bem


def _rand(n, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(n, dtype=torch.float64, generator=g) + 1j * torch.randn(n, dtype=torch.float64, generator=g)
    return x.to(torch.complex128).to(dev)


@pytest.mark.parametrize("npol", [1, 2])
def test_transposed_solve_adjoint_identity(cuda, npol):
    import torch
    from mnpbem_b200 import _native as nat
    cp = dimer()
    bem = _bem(cp, 620.0, "fp64")
    n = cp.n
    L = nat.lib()
    u = _rand(8 * n * npol, 1, cuda)
    v = _rand(8 * n * npol, 2, cuda)
    W1, W2 = bem.solve_device(v, npol)
    Sv = torch.cat([W1.reshape(-1), W2.reshape(-1)])
    scr = torch.empty(int(L.bem200_bem_solve_T_workspace_size(0, n, npol)), dtype=torch.uint8, device=cuda)
    STu = torch.empty_like(u)
    nat.call("bem200_bem_solve_T", 0, 0, n, npol, nat.ptr(bem._ws), nat.ptr(u), bem._eps_mode, bem._e1p, bem._e2p,
             nat.ptr(bem._nvec), bem.k, nat.ptr(STu), nat.ptr(scr), nat.stream_ptr())
    lhs = complex((STu * v).sum())
    rhs = complex((u * Sv).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(rhs), (lhs, rhs)


def test_transposed_operator_and_mixed_adjoint(cuda):
    """<A^T l, x> = <l, A x> for the FP64 operator; the refined complex64
    transposed solve reaches A^-T w to the refinement tolerance."""
    import torch
    from mnpbem_b200 import _native as nat
    from mnpbem_b200.shape import _transposed_solve
    cp = dimer()
    bem = _bem(cp, 620.0, "mixed")
    n, npol = cp.n, 1
    L = nat.lib()
    G = bem._G128
    x = _rand(8 * n, 3, cuda)
    lv = _rand(8 * n, 4, cuda)
    Ax = torch.empty_like(x)
    scr = torch.empty(int(L.bem200_bem_apply_workspace_size(n, npol)), dtype=torch.uint8, device=cuda)
    nat.call("bem200_bem_apply", n, npol, *[nat.ptr(m) for m in G], bem._eps_mode, bem._e1p, bem._e2p,
             nat.ptr(bem._nvec), bem.k, nat.ptr(x), ctypes.c_void_p(x.data_ptr() + 16 * 4 * n), None, nat.ptr(Ax),
             nat.ptr(scr), nat.stream_ptr())
    ATl = torch.empty_like(lv)
    scrT = torch.empty(int(L.bem200_bem_apply_T_workspace_size(n, npol)), dtype=torch.uint8, device=cuda)
    nat.call("bem200_bem_apply_T", n, npol, *[nat.ptr(m) for m in G], bem._eps_mode, bem._e1p, bem._e2p,
             nat.ptr(bem._nvec), bem.k, nat.ptr(lv), None, nat.ptr(ATl), nat.ptr(scrT), nat.stream_ptr())
    lhs, rhs = complex((ATl * x).sum()), complex((lv * Ax).sum())
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs), (lhs, rhs)
    w = _rand(8 * n, 5, cuda)
    lam, sweeps = _transposed_solve(bem, w, 1, tol=1e-12)
    nat.call("bem200_bem_apply_T", n, npol, *[nat.ptr(m) for m in G], bem._eps_mode, bem._e1p, bem._e2p,
             nat.ptr(bem._nvec), bem.k, nat.ptr(lam), nat.ptr(w), nat.ptr(ATl), nat.ptr(scrT), nat.stream_ptr())
    assert float(torch.linalg.vector_norm(ATl)) <= 1e-12 * float(torch.linalg.vector_norm(w)) and sweeps <= 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vertex_gradient_matches_reference_fd(cuda, precision):
    """The curved rod of shape_fd_rod.npz: the reverse-mode gradient along
    the fixture's directions equals the reference solver's own central
    differences (h = 1e-4 nm, whose noise is ~1e-7 relative)."""
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.shape import extinction_vertex_vjp, vertex_array
    g = golden("shape_fd_rod.npz")
    cp = shape_particle("rodbem")
    assert np.array_equal(vertex_array(cp), g["verts2"])
    bem = _bem(cp, float(g["enei"]), precision)
    ext, grad = extinction_vertex_vjp(bem, PlaneWaveRet(POL, DIR), float(g["enei"]))
    assert abs(ext[0] - float(g["ext"])) <= 1e-10 * abs(float(g["ext"]))
    dext = np.tensordot(g["D"], grad, axes=([1, 2], [0, 1]))
    err = np.max(np.abs(dext - g["dext"])) / np.max(np.abs(g["dext"]))
    assert err < 1e-6, (dext, g["dext"], err)


def _fd(cp, D, enei, pol, dirs, h=1e-3):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import perturbed
    exc = PlaneWaveRet(pol, dirs)
    out = []
    with refinement_of(cp):
        for s in (1.0, -1.0):
            q = perturbed(cp, s * h * D)
            out.append(BEMRet(q).cross_sections(exc, enei)["ext"])
    return (out[0] - out[1]) / (2 * h)


@pytest.mark.parametrize("mk,enei", [(sphere, 600.0), (dimer, 620.0), (lambda: shape_particle("ellbem"), 560.0)],
                         ids=["sphere284", "dimer568", "ellipsoid_flat"])
def test_vertex_gradient_matches_solver_fd(cuda, mk, enei):
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.shape import extinction_vertex_vjp, random_directions
    cp = mk()
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    bem = _bem(cp, enei, "fp64")
    wts = np.array([1.0, 0.5])
    ext, grad = extinction_vertex_vjp(bem, PlaneWaveRet(pol, dirs), enei, weights=wts)
    # ext is invariant under translation of the whole mesh
    assert np.all(np.abs(grad.sum(axis=0)) <= 1e-9 * np.abs(grad).sum(axis=0)), grad.sum(axis=0)
    # central differences with h = 1e-3 nm and the unperturbed refinement
    # pattern: truncation (h / radius)^2 ~ 1e-8, the FP64 solves' own noise
    # (~1e-12 of ext) / 2h ~ 1e-7 of the slope
    for D in random_directions(cp, 2, seed=7):
        ref = float(np.dot(wts, _fd(cp, D, enei, pol, dirs)))
        got = float(np.sum(grad * D))
        assert abs(got - ref) <= 2e-6 * max(abs(ref), 1e-3 * np.max(np.abs(ext))), (got, ref)
