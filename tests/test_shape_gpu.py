"""Vertex derivatives of the extinction (mnpbem_b200.shape) against central
finite differences of the whole solver along seeded random directions."""
import numpy as np
import pytest

from meshes import shape_particle

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0], [0, 0, 1.0]])
DIR = np.array([[0, 0, 1.0], [1.0, 0, 0]])
H = 1e-4      # nm, the finite-difference step of the check and of the assembly


def _fd(cp, D, enei, precision="fp64"):
    """Central difference of the full solve (new factors at each side)."""
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import perturbed
    exc = PlaneWaveRet(POL, DIR)
    out = []
    for d in D:
        e = []
        for s in (1.0, -1.0):
            q = perturbed(cp, s * H * d)
            sig, _ = BEMRet(q, precision=precision).solve(exc.potential(q, enei))
            e.append(np.asarray(exc.extinction(sig)))
        out.append((e[0] - e[1]) / (2 * H))
    return np.array(out)


@pytest.mark.parametrize("tag,enei", [("rodbem", 600.0), ("ellbem", 560.0)])
def test_directional_derivative_matches_central_differences(cuda, tag, enei):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import extinction_shape_derivative, random_directions
    cp = shape_particle(tag)
    D = random_directions(cp, 4, seed=11)
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp)
    ext, dext = extinction_shape_derivative(bem, exc, enei, D, h=H)
    sig, _ = BEMRet(cp).solve(exc.potential(cp, enei))
    np.testing.assert_allclose(ext, exc.extinction(sig), rtol=1e-12)
    fd = _fd(cp, D, enei)
    assert np.max(np.abs(dext - fd)) <= 1e-6 * np.max(np.abs(fd)), (dext, fd)


def test_mixed_matches_fp64(cuda):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import ShapeSensitivity, random_directions
    cp = shape_particle("cubebem")
    D = random_directions(cp, 3, seed=2)
    exc = PlaneWaveRet(POL, DIR)
    e64, d64 = ShapeSensitivity(BEMRet(cp), D, H).extinction(exc, 640.0)
    sens = ShapeSensitivity(BEMRet(cp, precision="mixed"), D, H)
    for enei in (640.0, 700.0):
        e32, d32 = sens.extinction(exc, enei)
        if enei == 640.0:
            assert np.max(np.abs(e32 - e64)) <= 1e-10 * np.max(np.abs(e64))
            assert np.max(np.abs(d32 - d64)) <= 1e-8 * np.max(np.abs(d64))
    fd = _fd(cp, D, 700.0)
    assert np.max(np.abs(d32 - fd)) <= 1e-6 * np.max(np.abs(fd))


def test_autograd_backward_and_jvp(cuda):
    import torch
    import torch.autograd.forward_ad as fwAD
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import ExtinctionShape, extinction_shape_derivative, random_directions
    cp = shape_particle("rodbem")
    D = random_directions(cp, 3, seed=5)
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp)
    _, dext = extinction_shape_derivative(bem, exc, 620.0, D, h=H)
    t = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    ext = ExtinctionShape.apply(t, bem, exc, 620.0, D)
    (ext * torch.tensor([1.0, 2.0], dtype=torch.float64)).sum().backward()
    # each call rebuilds the moved particles' Green functions, whose closed-surface
    # sums use FP64 atomics: last-bit differences, divided by the 2h step
    np.testing.assert_allclose(t.grad.numpy(), dext @ np.array([1.0, 2.0]), rtol=1e-8)
    tangent = torch.tensor([0.3, -1.0, 2.0], dtype=torch.float64)
    with fwAD.dual_level():
        out = ExtinctionShape.apply(fwAD.make_dual(torch.zeros(3, dtype=torch.float64), tangent), bem, exc, 620.0, D)
        jv = fwAD.unpack_dual(out).tangent
    np.testing.assert_allclose(jv.numpy(), tangent.numpy() @ dext, rtol=1e-8)
    # away from t = 0 a solver is built for the moved particle
    t1 = torch.tensor([0.2, 0.0, -0.1], dtype=torch.float64)
    e1 = ExtinctionShape.apply(t1, bem, exc, 620.0, D).numpy()
    from mnpbem_b200.shape import perturbed
    q = perturbed(cp, np.tensordot(t1.numpy(), D, axes=1))
    sig, _ = BEMRet(q).solve(exc.potential(q, 620.0))
    np.testing.assert_allclose(e1, exc.extinction(sig), rtol=1e-12)
