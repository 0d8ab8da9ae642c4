"""d(extinction)/d(eps) of the particle material (one extra solve with the
factors of the wavelength) against central finite differences of the FP64
solver, and through the torch.autograd wrapper."""
import numpy as np
import pytest

from meshes import DRUDE_AU
from mnpbem_b200.geometry import ComParticle, trisphere
from mnpbem_b200.materials import EpsConst, EpsDrude

pytestmark = pytest.mark.gpu
POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _sphere(metal, eps_b=1.0):
    return ComParticle([EpsConst(eps_b), metal], [trisphere(144, 20.0)], [[2, 1]], 1, interp="curv")


def _dimer(metal, eps_b=1.77):
    a, b = trisphere(144, 10.0), trisphere(144, 10.0)
    a.shift([-6.0, 0, 0])
    b.shift([6.0, 0, 0])
    return ComParticle([EpsConst(eps_b), metal], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")


def _ext(mk, eps_m, enei):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = mk(EpsConst(eps_m))
    exc = PlaneWaveRet(POL, DIR)
    sig, _ = BEMRet(cp).solve(exc.potential(cp, enei))
    return exc.extinction(sig)


@pytest.mark.parametrize("mk,enei", [(_sphere, 600.0), (_dimer, 620.0)], ids=["sphere", "dimer"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eps_gradient_matches_finite_differences(cuda, mk, enei, precision):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.adjoint import extinction_eps_gradient
    drude = EpsDrude(*DRUDE_AU)
    eps_m = complex(drude(enei)[0])
    cp = mk(drude)
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp, precision=precision)
    ext, grad = extinction_eps_gradient(bem, exc, enei, material=2)
    assert abs(ext[0] - _ext(mk, eps_m, enei)) / ext[0] < 1e-10
    h = 1e-4 * abs(eps_m)
    fd_u = (_ext(mk, eps_m + h, enei) - _ext(mk, eps_m - h, enei)) / (2 * h)
    fd_v = (_ext(mk, eps_m + 1j * h, enei) - _ext(mk, eps_m - 1j * h, enei)) / (2 * h)
    fd = np.array([fd_u, fd_v])
    assert np.linalg.norm(grad[0] - fd) / np.linalg.norm(fd) < 1e-6, (grad[0], fd)


def test_autograd_wrapper(cuda):
    import torch
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.adjoint import ExtinctionEps, extinction_eps_gradient
    drude = EpsDrude(*DRUDE_AU)
    cp = _sphere(drude)
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp)
    e = complex(drude(580.0)[0])
    x = torch.tensor([e.real, e.imag], dtype=torch.float64, requires_grad=True)
    ext = ExtinctionEps.apply(x, bem, exc, 580.0, 2)
    ext.sum().backward()
    _, grad = extinction_eps_gradient(bem, exc, 580.0, 2)
    assert np.allclose(x.grad.numpy(), grad[0], rtol=1e-12, atol=0)
