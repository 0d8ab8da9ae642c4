"""Wavelength sharding and the result gather of the multi-GPU sweep, run as
two gloo ranks on the CPU (the per-wavelength solver is a stand-in; the host
logic -- which rank solves which wavelength, the all-reduce of the results and
of the timing -- is what is tested)."""
import os

import numpy as np
import pytest

from mnpbem_b200.spectrum import shard


def test_shard_round_robin():
    assert shard(7, 0, 3) == [0, 3, 6] and shard(7, 1, 3) == [1, 4] and shard(7, 2, 3) == [2, 5]
    assert sorted(sum((shard(41, r, 4) for r in range(4)), [])) == list(range(41))
    assert shard(2, 3, 4) == []


def _rank_main(rank, world, port, enei, out_dir):
    import datetime
    import torch.distributed as dist
    from mnpbem_b200.spectrum import sweep_dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{}".format(port), rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    calls = []

    def fake_solve(lam):
        calls.append(lam)
        return np.array([lam, 2 * lam]), np.array([lam ** 0.5, 1.0 + rank])

    ext, sca, wall, mine = sweep_dist(fake_solve, enei, 2)
    np.savez(os.path.join(out_dir, "rank{}.npz".format(rank)), ext=ext, sca=sca, wall=wall, mine=np.array(mine),
             calls=np.array(calls))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sweep_gather_two_gloo_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    enei = np.linspace(400.0, 800.0, 9)
    port = 29000 + os.getpid() % 1000
    mp.start_processes(_rank_main, args=(world, port, enei, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [np.load(os.path.join(tmp_path, "rank{}.npz".format(r))) for r in range(world)]
    exp_ext = np.stack([enei, 2 * enei], axis=1)
    for r, d in enumerate(res):
        # every rank solved exactly its round-robin share ...
        np.testing.assert_array_equal(d["mine"], np.arange(r, len(enei), world))
        np.testing.assert_array_equal(d["calls"], enei[r::world])
        # ... and holds the full gathered spectrum
        np.testing.assert_array_equal(d["ext"], exp_ext)
        owner = np.arange(len(enei)) % world
        np.testing.assert_array_equal(d["sca"][:, 1], 1.0 + owner)
    assert res[0]["wall"] == res[1]["wall"]  # max over ranks on both
