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


class _Mesh:
    def __init__(self, n):
        self.n = n


def _fake_factory(calls):
    def factory(p, pol, dirs):
        def solve(enei):
            calls.append((p.n, float(enei)))
            k = len(pol)
            return np.array([p.n + enei, 2.0])[:k], np.array([enei, p.n])[:k]
        return solve
    return factory


def test_partition_units_covers_every_unit_once():
    from mnpbem_b200.sweep import partition_units
    sizes = [s[0] for s in UNEVEN_SHAPES]
    for world in (1, 2, 3, 8):
        parts = partition_units(sizes, 16, world)
        seen = np.zeros((len(sizes), 16), dtype=int)
        for p in parts:
            for m, lam in p.items():
                seen[m, lam] += 1
        assert np.all(seen == 1)
        load = [sum(len(lam) * float(sizes[m]) ** 3 for m, lam in p.items()) for p in parts]
        assert max(load) <= sum(load) / world + float(max(sizes)) ** 3


def test_solve_sweep_host_threads_with_a_stand_in_solver():
    """The worker threads and the (mesh, wavelength) plan of solve_sweep,
    with a stand-in solver: every unit once, results in place."""
    from mnpbem_b200.sweep import solve_sweep
    meshes = [_Mesh(n) for n in (284, 760, 1296)]
    enei = np.linspace(450.0, 900.0, 7)
    for schedule in ("interleave", "mesh"):
        calls = []
        r = solve_sweep(meshes, enei, [[1, 0, 0], [0, 1, 0]], [[0, 0, 1], [0, 0, 1]], workers=3, schedule=schedule,
                        solver_factory=_fake_factory(calls))
        assert sorted(calls) == sorted((m.n, float(e)) for m in meshes for e in enei)
        for mi, m in enumerate(meshes):
            np.testing.assert_array_equal(r["ext"][mi, :, 0], m.n + enei)
            np.testing.assert_array_equal(r["sca"][mi, :, 1], m.n)
        assert r["solves"] == 3 * 7 * 2
    # a share of the units only
    calls = []
    r = solve_sweep(meshes, enei, [[1, 0, 0]], [[0, 0, 1]], workers=2, units={1: np.array([0, 3])},
                    solver_factory=_fake_factory(calls))
    assert sorted(calls) == [(760, enei[0]), (760, enei[3])]
    assert r["solves"] == 2 and np.count_nonzero(r["ext"][:, :, 0]) == 2


def _dist_rank(rank, world, port, out_dir):
    import datetime
    import os
    import torch.distributed as dist
    from mnpbem_b200.sweep import solve_sweep_dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{}".format(port), rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    calls = []
    meshes = [_Mesh(n) for n in (284, 760, 1296, 2000)]
    enei = np.linspace(450.0, 900.0, 5)
    r = solve_sweep_dist(meshes, enei, [[1, 0, 0]], [[0, 0, 1]], workers=2, solver_factory=_fake_factory(calls))
    np.savez(os.path.join(out_dir, "rank{}.npz".format(rank)), ext=r["ext"], sca=r["sca"], solves=r["solves"],
             calls=np.array(calls))
    dist.destroy_process_group()


def test_uneven_sweep_two_gloo_ranks(tmp_path):
    import os
    import torch.multiprocessing as mp
    port = 29500 + os.getpid() % 400
    mp.start_processes(_dist_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [np.load(os.path.join(tmp_path, "rank{}.npz".format(r))) for r in range(2)]
    enei = np.linspace(450.0, 900.0, 5)
    sizes = (284, 760, 1296, 2000)
    all_calls = sorted(tuple(c) for d in res for c in d["calls"])
    assert all_calls == sorted((float(n), float(e)) for n in sizes for e in enei)   # each unit on one rank
    for d in res:
        for mi, n in enumerate(sizes):
            np.testing.assert_array_equal(d["ext"][mi, :, 0], n + enei)
        assert int(d["solves"]) == len(sizes) * len(enei)


def test_autotune_picks_the_fastest_schedule():
    """autotune_sweep with a stand-in solver whose time per call grows with
    the number of concurrent workers beyond 4: the 4-worker interleave wins."""
    import threading
    import time as _time
    from mnpbem_b200.sweep import autotune_sweep
    active = [0]
    lock = threading.Lock()

    def factory(p, pol, dirs):
        def solve(enei):
            with lock:
                active[0] += 1
                k = active[0]
            _time.sleep(0.004 * max(1, k - 3))      # contention above 4 concurrent solves
            with lock:
                active[0] -= 1
            return np.zeros(len(pol)), np.zeros(len(pol))
        return solve

    meshes = [_Mesh(n) for n in (284, 760, 1296, 2000, 2884, 3600, 4800, 5768)]
    best, rates = autotune_sweep(meshes, np.linspace(450, 900, 128), [[1, 0, 0]], [[0, 0, 1]], probe=16,
                                 candidates=((1, "interleave"), (4, "interleave"), (16, "interleave")),
                                 solver_factory=factory)
    assert set(rates) == {(1, "interleave"), (4, "interleave"), (16, "interleave")}
    assert best == (4, "interleave"), rates
