"""The GPU path on meshes from the reference's other generators: curved
quadrilaterals (trirod, tricube) and flat triangles (triellipsoid), against the
oracle and the reference BEMRet's own results (tests/golden/meshes.npz)."""
import numpy as np
import pytest

from conftest import golden
from meshes import rel, shape_particle
from oracle import green as og

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0], [0, 0, 1.0]])
DIR = np.array([[0, 0, 1.0], [1.0, 0, 0]])
TAGS = ["rodbem", "cubebem", "ellbem"]


@pytest.mark.parametrize("tag", TAGS)
def test_refinement_matches_oracle(cuda, tag):
    from mnpbem_b200.greenfun import CompGreenRet
    cp = shape_particle(tag)
    g = CompGreenRet(cp, cp)
    b = og.refine_all(cp)[0][0]
    r = g.refined
    n = r.nref
    order = np.lexsort((b.cols, b.rows))
    np.testing.assert_array_equal(r.row[:n].cpu().numpy(), b.rows[order])
    np.testing.assert_array_equal(r.col[:n].cpu().numpy(), b.cols[order])
    gg, fg = r.g[:n].cpu().numpy(), r.f[:n].cpu().numpy()
    go, fo = b.g[order], b.f[order]
    for m in range(gg.shape[1]):
        assert np.max(np.abs(gg[:, m] - go[:, m])) <= 1e-10 * np.max(np.abs(go[:, m])), ("g", m)
        assert np.max(np.abs(fg[:, :, m] - fo[:, :, m])) <= 1e-10 * np.max(np.abs(fo[:, :, m])), ("f", m)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tag", TAGS)
def test_bem_matches_reference(cuda, tag, precision):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    gl = golden("meshes.npz")
    cp = shape_particle(tag)
    bem = BEMRet(cp, precision=precision)
    exc = PlaneWaveRet(POL, DIR)
    tol = 1e-10 if precision == "fp64" else 1e-8
    for i, enei in enumerate(gl[tag + "_enei"]):
        sig, bem = bem.solve(exc.potential(cp, float(enei)))
        assert rel(exc.extinction(sig), gl[tag + "_ext"][i]) < tol
        assert rel(exc.scattering(sig)[0], gl[tag + "_sca"][i]) < tol
    assert rel(sig.sig2, gl[tag + "_sig2"]) < 1e2 * tol


def test_rod_config3_size(cuda):
    """The ~2400-face curved rod (trirod(20, 80, [41, 16, 31]), eps_b 1.77):
    mixed + refinement reproduces the fp64 extinction to 1e-8."""
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = shape_particle("rod2400")
    assert cp.n == 2400
    exc = PlaneWaveRet(POL[:1], DIR[:1])
    out = []
    for precision in ("fp64", "mixed"):
        bem = BEMRet(cp, precision=precision)
        sig, _ = bem.solve(exc.potential(cp, 700.0))
        out.append(exc.extinction(sig))
    assert abs(out[1] - out[0]) / abs(out[0]) < 1e-8


def test_uneven_sweep_two_workers(cuda):
    """Three small meshes of the uneven batch (sphere, ellipsoid, rod) swept
    over 3 wavelengths x 2 polarisations on two streams, both schedules:
    the same to 1e-12 (each BEMRet sums its closed-surface corrections with FP64
    atomics, so separately built solvers differ in the last bits) and within
    1e-8 of fp64 solves."""
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.sweep import uneven_meshes, solve_sweep
    shapes = ((284, "sphere", 144), (760, "ellipsoid", 382), (1296, "rod", (25, 14, 29)))
    ms = uneven_meshes(3, shapes=shapes)
    parts = [m["p"] for m in ms]
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    enei = np.array([480.0, 610.0, 870.0])
    r2 = solve_sweep(parts, enei, pol, dirs, workers=2)
    r1 = solve_sweep(parts, enei, pol, dirs, workers=2, schedule="mesh")
    assert r2["solves"] == 18
    assert rel(r2["ext"], r1["ext"]) < 1e-12
    assert rel(r2["sca"], r1["sca"]) < 1e-12
    exc = PlaneWaveRet(pol, dirs)
    for m, cp in enumerate(parts):
        ref = BEMRet(cp)
        for i, e in enumerate(enei):
            sig, _ = ref.solve(exc.potential(cp, float(e)))
            assert rel(r2["ext"][m, i], exc.extinction(sig)) < 1e-8
            assert rel(r2["sca"][m, i], exc.scattering(sig)[0]) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rod_matches_mnpbem17(cuda, precision):
    """The gold rod trirod(10, 40, [15, 15, 15]) (588 curved faces, vacuum,
    tabulated gold, x-pol along +z and z-pol along +x) against MNPBEM17
    (MATLAB) at 5 of the 41 wavelengths of the reference's validation CSV."""
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.geometry import ComParticle, trirod
    from mnpbem_b200.materials import EpsConst, EpsValues
    g = golden("matlab_rod.npz")
    cp = ComParticle([EpsConst(1.0), EpsValues(dict(zip(g["enei"], g["eps_gold"])))],
                     [trirod(10.0, 40.0, [15, 15, 15])], [[2, 1]], 1, interp="curv")
    bem = BEMRet(cp, precision=precision)
    exc = PlaneWaveRet(POL, DIR)
    for i in (0, 10, 20, 30, 40):
        sig, bem = bem.solve(exc.potential(cp, float(g["enei"][i])))
        ext, sca = exc.extinction(sig), exc.scattering(sig)[0]
        got = np.array([ext[0], sca[0], ext[1], sca[1]])
        assert np.max(np.abs(got - g["matlab"][i]) / np.abs(g["matlab"][i])) < 1e-9, (i, got, g["matlab"][i])
