"""The restated mesh generators (triellipsoid, trispheresegment, trirod,
tricube) against the reference's own output (tests/golden/meshes.npz), and the
oracle BEM on a curved rod and a rounded cube (quadrilateral faces) against
the reference BEMRet."""
import numpy as np
import pytest

from conftest import golden
from meshes import MESH_CASES, face_nodes, rel, shape_particle
from mnpbem_b200 import geometry


@pytest.mark.parametrize("tag", sorted(MESH_CASES))
def test_generator_matches_reference(tag):
    g = golden("meshes.npz")
    name, args, kw = MESH_CASES[tag]
    p = getattr(geometry, name)(*args, **kw)
    assert p.nfaces == int(g[tag + "_nfaces"])
    assert p.nverts == int(g[tag + "_nverts"])
    assert int(np.sum(np.isnan(p.faces[:, 3]))) == int(g[tag + "_ntri"])
    ind = g[tag + "_ind"]
    # same arithmetic in the same order: the face arrays agree to the bit
    for a in ("pos", "nvec", "tvec1", "area"):
        np.testing.assert_array_equal(getattr(p, a)[ind], g[tag + "_" + a], err_msg=a)
    np.testing.assert_array_equal(p.bradius()[ind], g[tag + "_bradius"])
    np.testing.assert_array_equal(face_nodes(p)[ind], g[tag + "_nodes"])
    assert np.sum(p.area) == pytest.approx(float(g[tag + "_area_sum"]), rel=1e-14)


def test_tricube_face_count():
    # 6 (n - 1)^2 quads less the faces the area cut-off of clean() removes
    assert geometry.tricube(66, 100.0).nfaces == 25344
    assert geometry.tricube(6, 40.0).nfaces == 150


def test_clean_and_select():
    # two unit squares sharing an edge, given with duplicated vertices
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [1, 0, 0], [2, 0, 0], [2, 1, 0], [1, 1, 0.0]])
    f = np.array([[0, 1, 2, 3], [4, 5, 6, 7.0]])
    p = geometry.Particle(v, f).clean()
    assert p.nverts == 6 and p.nfaces == 2
    a, b = p.select(index=[1])
    assert a.nfaces == 1 and a.nverts == 4 and b.nfaces == 1
    np.testing.assert_allclose(a.pos, [[1.5, 0.5, 0]])
    # a quad with a repeated corner becomes a triangle in its original winding
    q = geometry.Particle(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0.0]]), np.array([[0, 1, 1, 2.0]])).clean()
    np.testing.assert_array_equal(q.faces[0, :3], [0, 1, 2])
    assert np.isnan(q.faces[0, 3])


def test_flip_keeps_normals_outward():
    p = geometry.trirod(12.0, 30.0, [9, 5, 5], interp="curv")
    q = p.flip(2)
    np.testing.assert_allclose(q.pos[:, 2], -p.pos[:, 2], atol=1e-13)
    # outward: n . (pos - centre) > 0 on both
    assert np.all(np.sum(q.nvec * q.pos, axis=1) > 0)


@pytest.mark.parametrize("tag", ["rodbem", "cubebem", "ellbem"])
def test_oracle_bem_on_quad_meshes(tag):
    from oracle.pipeline import OracleBEM
    g = golden("meshes.npz")
    cp = shape_particle(tag)
    assert cp.n == int(g[tag + "_nfaces"])
    ob = OracleBEM(cp)
    pol = [[1.0, 0, 0], [0, 0, 1.0]]
    dirs = [[0, 0, 1.0], [1.0, 0, 0]]
    for i, e in enumerate(g[tag + "_enei"]):
        out = ob.solve(float(e), pol, dirs)
        assert rel(out["ext"], g[tag + "_ext"][i]) < 1e-11
        assert rel(out["sca"], g[tag + "_sca"][i]) < 1e-11
    assert rel(out["sig2"], g[tag + "_sig2"]) < 1e-10


def test_oracle_rod_matches_mnpbem17_and_reference():
    """trirod(10, 40, [15, 15, 15]) (588 curved faces), vacuum, tabulated gold,
    x-pol along +z and z-pol along +x: the oracle reproduces MNPBEM17 (MATLAB)
    to the 11 digits stored in the reference's validation CSV
    (validation/03_bemret/rod/data/bemret_matlab.csv).  The reference
    Python package of this checkout does too; its own committed CSV
    (bemret_python.csv) is older and differs from both by up to 7e-6."""
    from mnpbem_b200.geometry import ComParticle, trirod
    from mnpbem_b200.materials import EpsConst, EpsValues
    from oracle.pipeline import OracleBEM
    g = golden("matlab_rod.npz")
    table = dict(zip(g["enei"], g["eps_gold"]))
    cp = ComParticle([EpsConst(1.0), EpsValues(table)], [trirod(10.0, 40.0, [15, 15, 15])], [[2, 1]], 1,
                     interp="curv")
    assert cp.n == 588
    ob = OracleBEM(cp)
    pol = [[1.0, 0, 0], [0, 0, 1.0]]
    dirs = [[0, 0, 1.0], [1.0, 0, 0]]
    for i in (0, 20, 40):
        out = ob.solve(float(g["enei"][i]), pol, dirs)
        got = np.array([out["ext"][0], out["sca"][0], out["ext"][1], out["sca"][1]])
        assert np.max(np.abs(got - g["matlab"][i]) / np.abs(g["matlab"][i])) < 5e-10, i
        assert np.max(np.abs(got - g["python"][i]) / np.abs(g["python"][i])) < 1e-5, i


def test_planewave_field_matches_reference():
    from mnpbem_b200.planewave import PlaneWaveRet
    g = golden("planewave_field.npz")
    cp = shape_particle("rodbem")
    exc = PlaneWaveRet([[1.0, 0, 0], [0, 0, 1.0]], [[0, 0, 1.0], [1.0, 0, 0]])
    for inout in (1, 2):
        f = exc.field(cp, 600.0, inout=inout)
        np.testing.assert_allclose(f.e, g["e%d" % inout], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(f.h, g["h%d" % inout], rtol=1e-14, atol=1e-15)
