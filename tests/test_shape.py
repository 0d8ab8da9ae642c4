"""Host side of the vertex derivatives: the vertex space and moved particles (no GPU)."""
import numpy as np

from meshes import shape_particle
from mnpbem_b200.shape import perturbed, random_directions, vertex_array


def test_zero_move_reproduces_geometry():
    for tag in ("rodbem", "ellbem"):
        cp = shape_particle(tag)
        q = perturbed(cp, np.zeros_like(vertex_array(cp)))
        for a in ("pos", "nvec", "tvec1", "area"):
            np.testing.assert_array_equal(getattr(q, a), getattr(cp, a))
        assert q is not cp and q.p[0] is not cp.p[0]


def test_vertex_space_and_translation():
    cp = shape_particle("rodbem")          # curved: the space is verts2
    v = vertex_array(cp)
    assert v.shape == cp.p[0].verts2.shape
    q = perturbed(cp, np.tile([0.5, -0.25, 1.0], (len(v), 1)))
    np.testing.assert_allclose(q.pos - cp.pos, np.tile([0.5, -0.25, 1.0], (cp.n, 1)), atol=1e-12)
    np.testing.assert_allclose(q.area, cp.area, rtol=1e-12)
    np.testing.assert_allclose(q.nvec, cp.nvec, atol=1e-12)
    # the original is untouched
    np.testing.assert_array_equal(vertex_array(cp), v)


def test_flat_centroids_move_linearly():
    cp = shape_particle("ellbem")          # flat: the space is verts, pos = corner mean
    d = random_directions(cp, 1, seed=4)[0]
    q = perturbed(cp, 1e-3 * d)
    f = cp.p[0].faces[:, :3].astype(int)
    np.testing.assert_allclose(q.pos - cp.pos, 1e-3 * d[f].mean(axis=1), atol=1e-15)


def test_random_directions_are_unit_and_seeded():
    cp = shape_particle("cubebem")
    d = random_directions(cp, 5, seed=1)
    assert d.shape == (5,) + vertex_array(cp).shape
    np.testing.assert_allclose(np.sqrt(np.sum(d * d, axis=(1, 2))), 1.0)
    np.testing.assert_array_equal(d, random_directions(cp, 5, seed=1))


def test_autograd_plumbing_with_a_stand_in_derivative(monkeypatch):
    """The torch.autograd.Function (backward and forward-mode jvp) around a
    stand-in for the GPU derivative: ext = (1, 2), d ext / d t = J."""
    import torch
    import torch.autograd.forward_ad as fwAD
    from mnpbem_b200 import shape
    J = np.array([[1.0, -2.0], [0.5, 3.0], [4.0, 0.25]])
    monkeypatch.setattr(shape, "extinction_shape_derivative",
                        lambda bem, exc, enei, D, h: (np.array([1.0, 2.0]), J))
    D = np.zeros((3, 5, 3))
    t = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    ext = shape.ExtinctionShape.apply(t, None, None, 600.0, D)
    np.testing.assert_array_equal(ext.detach().numpy(), [1.0, 2.0])
    (ext * torch.tensor([3.0, -1.0], dtype=torch.float64)).sum().backward()
    np.testing.assert_allclose(t.grad.numpy(), J @ np.array([3.0, -1.0]))
    tangent = torch.tensor([1.0, 0.0, -2.0], dtype=torch.float64)
    with fwAD.dual_level():
        out = shape.ExtinctionShape.apply(fwAD.make_dual(torch.zeros(3, dtype=torch.float64), tangent), None, None,
                                          600.0, D)
        jv = fwAD.unpack_dual(out).tangent
    np.testing.assert_allclose(jv.numpy(), tangent.numpy() @ J)
