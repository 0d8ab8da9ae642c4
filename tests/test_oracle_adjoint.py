"""The oracle's transposed BEM solve and reverse-mode derivatives (CPU): the
adjoint identities, and one transposed solve against one tangent solve per
direction and against finite differences of the full solve."""
import numpy as np
import pytest

from meshes import rel, shape_particle
from oracle import adjoint as oad
from oracle import bem as obem

POL = np.array([[1.0, 0, 0], [0, 0, 1.0]])
DIR = np.array([[0, 0, 1.0], [1.0, 0, 0]])


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("tag", ["rodbem", "ellbem"])
def test_transposed_solve_and_operator(tag):
    cp = shape_particle(tag)
    enei = 600.0
    (G1, G2, H1, H2, e1, e2), st, _ = oad._state(cp, enei, POL, DIR)
    n, p = cp.n, 2
    rng = np.random.default_rng(3)
    u = (_rand(rng, n, p), _rand(rng, n, p), _rand(rng, n, 3, p), _rand(rng, n, 3, p))      # unknowns
    v = (_rand(rng, n, p), _rand(rng, n, 3, p), _rand(rng, n, 3, p), _rand(rng, n, p))      # equations
    # <S^T u, v> = <u, S v>
    lhs = oad._pair(oad.bem_solve_T(st, *u), v)
    rhs = oad._pair(u, obem.bem_solve(st, *v))
    assert rel(lhs, rhs) < 1e-10
    # <A^T v, x> = <v, A x>
    x = u
    Ax = obem.bem_operator(G1, G2, H1, H2, e1, e2, cp.nvec, enei, *x)
    assert rel(oad._pair(oad.bem_operator_T(G1, G2, H1, H2, e1, e2, cp.nvec, enei, *v), x), oad._pair(v, Ax)) < 1e-10
    # A^T S^T u = u
    back = oad.bem_operator_T(G1, G2, H1, H2, e1, e2, cp.nvec, enei, *oad.bem_solve_T(st, *u))
    for b_, u_ in zip(back, u):
        assert rel(b_, u_) < 1e-8


def test_extinction_weights_reproduce_extinction():
    from oracle import farfield as off
    cp = shape_particle("cubebem")
    enei = 640.0
    _, st, rhs = oad._state(cp, enei, POL, DIR)
    x = obem.bem_solve(st, *rhs)
    z = oad._pair(oad.extinction_weights(cp, enei, POL, DIR), x)
    k = complex(np.asarray(cp.eps[0](enei)[1]).ravel()[0])
    ext = off.extinction(cp, x[0], x[1], x[2], x[3], enei, POL, DIR)
    assert rel(np.real(4 * np.pi / k * np.imag(z)), ext) < 1e-12


def test_reverse_mode_matches_tangent_and_finite_differences():
    from mnpbem_b200.shape import perturbed, random_directions
    from oracle.pipeline import OracleBEM
    cp = shape_particle("rodbem")
    enei = 600.0
    D = random_directions(cp, 3, seed=7)
    ext, drev, _ = oad.reverse_directional(cp, enei, POL, DIR, D)
    dtan = oad.tangent_directional(cp, enei, POL, DIR, D)
    assert rel(drev, dtan) < 1e-9
    h = 1e-4
    fd = []
    for d in D:
        e = [OracleBEM(q).solve(enei, POL, DIR)["ext"] for q in (perturbed(cp, h * d), perturbed(cp, -h * d))]
        fd.append((e[0] - e[1]) / (2 * h))
    assert rel(drev, np.array(fd)) < 1e-6
    assert rel(ext, OracleBEM(cp).solve(enei, POL, DIR)["ext"]) < 1e-12
