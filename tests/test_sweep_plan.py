"""Host-side scheduling of the uneven-mesh sweep (no GPU)."""
import numpy as np

from mnpbem_b200.sweep import UNEVEN_SHAPES, lpt, sweep_plan


def test_interleave_covers_every_pair_once():
    sizes = [s[0] for s in UNEVEN_SHAPES]
    for workers in (1, 2, 3, 4):
        plan = sweep_plan(sizes, 128, workers)
        seen = np.zeros((len(sizes), 128), dtype=int)
        for w in plan:
            for m, lam in w:
                seen[m, lam] += 1
        assert np.all(seen == 1)
        # equal load: every worker has every mesh
        assert all(sorted(m for m, _ in w) == list(range(len(sizes))) for w in plan)
        # workers start on different meshes
        assert len({w[0][0] for w in plan}) == workers


def test_mesh_schedule_is_lpt():
    sizes = [s[0] for s in UNEVEN_SHAPES]
    plan = sweep_plan(sizes, 5, 2, "mesh")
    assert [m for m, _ in plan[0]] == [7]
    assert sorted(m for m, _ in plan[1]) == list(range(7))
    assert lpt([3.0, 3.0, 2.0, 2.0, 2.0], 2) == [[0, 2, 4], [1, 3]]


def test_uneven_meshes_face_counts():
    from mnpbem_b200.sweep import uneven_meshes
    ms = uneven_meshes(0)
    assert [m["n"] for m in ms] == [284, 760, 1296, 2000, 2884, 3600, 4800, 5768]
    assert {m["shape"] for m in ms} == {"sphere", "ellipsoid", "rod"}
    assert {m["metal"] for m in ms} <= {"gold", "silver"}
