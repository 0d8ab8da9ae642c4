"""The large-mesh configuration at full size: the rounded gold cube
tricube(66, 100 nm, e = 0.25) (25,344 curved quads), vacuum, 700 nm,
x-polarised plane wave along +z.

* BEMRetIter with the FP64 dense operator and the complex64 tensor-core LU as
  preconditioner (tol 1e-8) against BEMRetIter with the H-matrix operator
  (reference BEMRetIter(hmatrix=True), mnpbem/bem/bem_ret_iter.py:455-1744;
  htol 1e-6, tol 1e-6): the extinctions agree to the H-matrix tolerance;
* the reverse-mode vertex gradient at this size (Green and derivative tiles
  recomputed in the backward pass, no n x n x 3 storage): its sum over the
  vertices vanishes (ext is invariant under translation), and it matches
  central differences of full solves along a seeded direction, with the
  refinement pattern of the unperturbed mesh.

Each solver is released before the next is built (the dense path holds
about 100 GB)."""
import gc

import numpy as np
import pytest

from meshes import refinement_of

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])
ENEI = 700.0


def _cube():
    from mnpbem_b200 import ComParticle, EpsConst, EpsDrude
    from mnpbem_b200.geometry import tricube
    return ComParticle([EpsConst(1.0), EpsDrude(9.84, 9.0, 0.067)], [tricube(66, 100.0, 0.25, interp="curv")],
                       [[2, 1]], 1, interp="curv")


def _release():
    import torch
    gc.collect()
    torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def cube():
    return _cube()


def test_cube25k_dense_preconditioned_vs_hmatrix(cuda, cube):
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.bem_iter import BEMRetIter
    exc = PlaneWaveRet(POL, DIR)
    assert cube.n == 25344
    bem = BEMRetIter(cube, tol=1e-8, maxit=200)
    sig, bem = bem.solve(exc.potential(cube, ENEI))
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-8, bem.info()
    ext_dense = exc.extinction(sig)
    del bem, sig
    _release()
    hb = BEMRetIter(cube, hmatrix=True, cleaf=64, htol=1e-6, tol=1e-6, maxit=400)
    sig, hb = hb.solve(exc.potential(cube, ENEI))
    it, rr, fl = hb.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-6, hb.info()
    ext_h = exc.extinction(sig)
    del hb, sig
    _release()
    assert abs(ext_h - ext_dense) <= 1e-5 * abs(ext_dense), (ext_h, ext_dense)


def test_cube25k_vertex_gradient_vs_fd(cuda, cube):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.shape import extinction_vertex_vjp, perturbed, random_directions
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cube, precision="mixed")
    ext, grad = extinction_vertex_vjp(bem, exc, ENEI)
    del bem
    _release()
    tsum = np.abs(grad.sum(axis=0))
    assert np.all(tsum <= 1e-7 * np.abs(grad).sum(axis=0)), tsum
    D = random_directions(cube, 1, seed=3)[0]
    h = 1e-3  # the solver's own noise (~1e-12 of ext) sets the step at this size
    side = []
    with refinement_of(cube):
        for s in (1.0, -1.0):
            q = perturbed(cube, s * h * D)
            b = BEMRet(q, precision="mixed")
            side.append(float(b.cross_sections(exc, ENEI)["ext"][0]))
            del b, q
            _release()
    fd = (side[0] - side[1]) / (2 * h)
    got = float(np.sum(grad * D))
    assert abs(got - fd) <= 2e-4 * abs(fd) + 1e-8 * abs(ext[0]), (got, fd)
