"""Host geometry vs the reference meshes (golden vectors from the reference)."""
import numpy as np

from conftest import golden
from mnpbem_b200.geometry import Particle, trisphere
from mnpbem_b200.quadrature import QuadFace, lgl_nodes


def test_quadrature_sums():
    q = QuadFace()
    assert len(q.x) == 28 and abs(q.w.sum() - 1) < 1e-14
    assert len(q.x3) == 144 and abs(q.w3.sum() - 1) < 1e-14
    assert len(q.x4) == 192 and abs(q.w4.sum() - 4) < 1e-13
    x, w = lgl_nodes(5)
    assert abs(w.sum() - 2) < 1e-14 and x[0] == 1.0


def test_quadrature_exactness():
    # the 28-point rule integrates x^a y^b exactly up to degree 11 (sum w = 1 <-> area 1/2)
    from math import factorial
    q = QuadFace()
    for a in range(0, 6):
        for b in range(0, 6 - a):
            exact = factorial(a) * factorial(b) / factorial(a + b + 2) * 2  # normalised by area 1/2
            assert abs(np.sum(q.w * q.x ** a * q.y ** b) - exact) < 1e-13


def _cmp(tag, p, g):
    ind = g[tag + "_ind"]
    for a in ("pos", "nvec", "tvec1", "tvec2", "area"):
        np.testing.assert_allclose(getattr(p, a)[ind], g[tag + "_" + a], rtol=0, atol=1e-13)
    np.testing.assert_allclose(p.bradius()[ind], g[tag + "_bradius"], rtol=0, atol=1e-13)
    sub = ind[:12]
    qp, qw, qr = p.quadpol(sub)
    np.testing.assert_allclose(qp, g[tag + "_quadpol_pos"], atol=1e-13)
    np.testing.assert_allclose(qw, g[tag + "_quadpol_w"], atol=1e-15)
    np.testing.assert_array_equal(qr, g[tag + "_quadpol_row"])
    qp, qw, qr = p.quad_integration(sub)
    np.testing.assert_allclose(qp, g[tag + "_quad_pos"], atol=1e-13)
    np.testing.assert_allclose(np.asarray(qw.sum(axis=0)).ravel(), g[tag + "_quad_w"], atol=1e-15)


def test_trisphere_matches_reference():
    g = golden("geom_spheres.npz")
    _cmp("s144", trisphere(144, 20.0), g)
    _cmp("s1444", trisphere(1444, 40.0), g)


def test_trisphere_topology():
    p = trisphere(144, 20.0)
    assert p.nfaces == 284 and p.verts.shape == (144, 3)
    assert abs(p.area.sum() - np.pi * 20.0 ** 2) / (np.pi * 400) < 2e-3
    # outward normals
    assert np.all(np.sum(p.nvec * p.pos, axis=1) > 0)


def test_flat_and_quad_faces():
    # unit cube made of quads: flat areas, centroids and quadrature weights
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    f = np.array([[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7]], float)
    p = Particle(v, f)
    np.testing.assert_allclose(p.area, np.ones(6), atol=1e-14)
    qp, qw, qr = p.quad_integration()
    np.testing.assert_allclose(np.asarray(qw.sum(axis=1)).ravel(), np.ones(6), atol=1e-14)
    pp, pw, pr = p.quadpol()
    np.testing.assert_allclose(np.bincount(pr, weights=pw), np.ones(6), atol=1e-12)
    c = p.curved()
    np.testing.assert_allclose(c.area, np.ones(6), atol=1e-12)


def test_eps_tables_match_reference():
    """EpsTable by name reads the tables the reference ships (regenerated by
    mnpbem_b200/data/make_data.py) and interpolates them like the reference."""
    import pytest
    from conftest import golden
    from mnpbem_b200.materials import EpsTable
    g = golden("eps_tables.npz")
    for name in ("gold", "silver", "goldpalik", "silverpalik", "copperpalik"):
        eps, k = EpsTable(name + ".dat")(g[name + "_enei"])
        np.testing.assert_allclose(eps, g[name + "_eps"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(k, g[name + "_k"], rtol=1e-14, atol=0)
    with pytest.raises(ValueError):
        EpsTable("gold.dat")(5000.0)
    with pytest.raises(FileNotFoundError):
        EpsTable("unobtainium.dat")


def test_drude_presets_match_reference():
    from conftest import golden
    from mnpbem_b200.materials import EpsDrude
    g = golden("eps_tables.npz")
    for metal in ("gold", "silver", "aluminum"):
        m = getattr(EpsDrude, metal)()
        np.testing.assert_allclose([m.eps0, m.wp, m.gammad], g["drude_" + metal], rtol=1e-15)
    assert EpsDrude.from_name("Au").wp == EpsDrude.gold().wp


def test_rot_and_compound_editing_match_reference():
    from conftest import golden
    from mnpbem_b200.geometry import ComParticle, trisphere
    from mnpbem_b200.materials import EpsConst, EpsDrude
    g = golden("editing.npz")
    a, b = trisphere(60, 10.0), trisphere(32, 6.0)
    a.rot(30.0, [1.0, 1.0, 0.0])
    b.shift([9.0, 0.0, 0.0])
    np.testing.assert_allclose(a.pos, g["rot_pos"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(a.nvec, g["rot_nvec"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(a.area, g["rot_area"], rtol=1e-13)
    p = ComParticle([EpsConst(1.0), EpsDrude(9.84, 9.0, 0.067)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")
    p.shift([1.0, -2.0, 0.5]).scale(1.5).rot(45.0, [0.0, 0.0, 1.0])
    np.testing.assert_allclose(p.pos, g["cp_pos"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(p.nvec, g["cp_nvec"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(p.area, g["cp_area"], rtol=1e-13)
    part, local = p.ipart(g["ipart_ind"])
    np.testing.assert_array_equal(part, g["ipart_part"])
    np.testing.assert_array_equal(local, g["ipart_local"])
