"""GPU refinement + Green assembly (libbem200) against the CPU oracle."""
import numpy as np
import pytest

from meshes import dimer, rel, sphere
from oracle import green as og

pytestmark = pytest.mark.gpu


def _gpu_refined(g):
    r = g.refined
    n = r.nref
    return (r.row[:n].cpu().numpy(), r.col[:n].cpu().numpy(), r.kind[:n].cpu().numpy(),
            r.g[:n].cpu().numpy(), r.f[:n].cpu().numpy())


def _oracle_global(cp, blocks):
    off = cp.offsets
    rows, cols, kinds, gs, fs = [], [], [], [], []
    for a in range(len(cp.p)):
        for b in range(len(cp.p)):
            blk = blocks[a][b]
            rows.append(blk.rows + off[a])
            cols.append(blk.cols + off[b])
            kinds.append(blk.kind)
            gs.append(blk.g)
            fs.append(blk.f)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    order = np.lexsort((cols, rows))
    return (rows[order], cols[order], np.concatenate(kinds)[order], np.concatenate(gs)[order],
            np.concatenate(fs)[order])


@pytest.mark.parametrize("mk", [sphere, dimer], ids=["sphere284", "dimer568"])
def test_refinement_matches_oracle(cuda, mk):
    from mnpbem_b200.greenfun import CompGreenRet
    cp = mk()
    g = CompGreenRet(cp, cp)
    ro, co, ko, go, fo = _oracle_global(cp, og.refine_all(cp))
    rg, cg, kg, gg, fg = _gpu_refined(g)
    np.testing.assert_array_equal(rg, ro)
    np.testing.assert_array_equal(cg, co)
    np.testing.assert_array_equal(kg, ko)
    # polar points sit 5e-7 face radii from the centroid: the positions cancel
    # against the centroid, so both sides are only accurate to ~1e-11 there
    for m in range(gg.shape[1]):
        scale_g = np.max(np.abs(go[:, m]))
        scale_f = np.max(np.abs(fo[:, :, m]))
        assert np.max(np.abs(gg[:, m] - go[:, m])) <= 1e-10 * scale_g, ("g", m)
        assert np.max(np.abs(fg[:, :, m] - fo[:, :, m])) <= 1e-10 * scale_f, ("f", m)


@pytest.mark.parametrize("mk,enei", [(sphere, 600.0), (dimer, 650.0)], ids=["sphere284", "dimer568"])
def test_bem_matrices_match_oracle(cuda, mk, enei):
    from mnpbem_b200.greenfun import CompGreenRet
    cp = mk()
    g = CompGreenRet(cp, cp)
    ref = og.bem_matrices(cp, og.refine_all(cp), enei)
    got = g.bem_matrices(enei, dtype="c128")
    for name, a, b in zip(("G1", "G2", "H1", "H2"), got, ref):
        assert rel(a.cpu().numpy(), b) < 1e-10, name
    got64 = g.bem_matrices(enei, dtype="c64")
    for name, a, b in zip(("G1", "G2", "H1", "H2"), got64, ref):
        assert rel(a.cpu().numpy(), b) < 2e-7, name


def test_eval_region_pairs(cuda):
    from mnpbem_b200.greenfun import CompGreenRet
    cp = dimer()
    g = CompGreenRet(cp, cp)
    blocks = og.refine_all(cp)
    for (i, j) in ((0, 0), (1, 1), (1, 0)):
        for key in ("G", "H1", "H2", "F"):
            ref = og.green_region(cp, blocks, i, j, "F" if key == "F" else key, 700.0)
            got = g.eval(i, j, key, 700.0)
            if isinstance(ref, int):
                assert isinstance(got, int) and got == 0
            else:
                assert rel(got, ref) < 1e-10, (i, j, key)
