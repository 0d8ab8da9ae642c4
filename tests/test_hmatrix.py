"""H-matrix host side (cluster tree, block partition) and the oracle ACA,
against the reference's own trees, block lists and ACA ranks
(tests/golden/hmat_trees.npz, made by make_golden.py)."""
import numpy as np
import pytest

from conftest import golden
from meshes import DRUDE_AU, dimer
from mnpbem_b200.geometry import ComParticle, trisphere
from mnpbem_b200.hmatrix import ClusterTree, block_partition, make_kaware_fadmiss, particle_index
from mnpbem_b200.materials import EpsConst, EpsDrude
from oracle import hmatrix as oh
from oracle.pipeline import OracleBEM

ENEI = 600.0


def _case(tag):
    if tag == "s":
        cp = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20.0)], [[2, 1]], 1, interp="curv")
        return cp, 32, 1.0
    return dimer(), 64, 2.5


@pytest.mark.parametrize("tag", ["s", "d"])
def test_cluster_tree_matches_reference(tag):
    g = golden("hmat_trees.npz")
    cp, cleaf, _ = _case(tag)
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    np.testing.assert_array_equal(t.son, g[tag + "_son"])
    np.testing.assert_array_equal(t.cind, g[tag + "_cind"])
    np.testing.assert_array_equal(t.ind, g[tag + "_ind"])
    np.testing.assert_array_equal(t.ipart, g[tag + "_ipart"])
    np.testing.assert_allclose(t.rad, g[tag + "_rad"], rtol=1e-14)
    np.testing.assert_allclose(t.mid, g[tag + "_mid"], rtol=1e-14, atol=1e-13)


@pytest.mark.parametrize("tag", ["s", "d"])
def test_block_partition_matches_reference(tag):
    g = golden("hmat_trees.npz")
    cp, cleaf, eta = _case(tag)
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    dense, low = block_partition(t, make_kaware_fadmiss(2 * np.pi / ENEI, eta0=eta))
    np.testing.assert_array_equal(np.array(dense, dtype=np.int64).reshape(-1, 2), np.stack([g[tag + "_row1"],
                                                                                          g[tag + "_col1"]], 1))
    np.testing.assert_array_equal(np.array(low, dtype=np.int64).reshape(-1, 2), np.stack([g[tag + "_row2"],
                                                                                        g[tag + "_col2"]], 1))


@pytest.mark.parametrize("tag", ["s", "d"])
def test_oracle_aca_matches_reference_ranks(tag):
    g = golden("hmat_trees.npz")
    cp, cleaf, eta = _case(tag)
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    dense, low = block_partition(t, make_kaware_fadmiss(2 * np.pi / ENEI, eta0=eta))
    G1 = OracleBEM(cp).matrices(ENEI)[0]
    full, ranks = oh.hmatrix_full(t, dense, low, G1, htol=1e-6, kmax=100)
    np.testing.assert_array_equal(ranks, g[tag + "_ranks"])
    err = np.linalg.norm(full - G1) / np.linalg.norm(G1)
    assert abs(err - float(g[tag + "_aca_err"])) <= 1e-3 * float(g[tag + "_aca_err"]) + 1e-12
