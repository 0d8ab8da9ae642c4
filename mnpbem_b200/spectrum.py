"""Wavelength sweeps of the retarded BEM solve, on one GPU or one process per GPU.

The path shards over independent wavelengths with no exchange but the final
gather of the (n_lambda x n_pol) cross sections, exactly the reference's
production parallel axis (mnpbem/utils/multi_gpu.py:148-260,
solve_spectrum_multi_gpu: wavelength i goes to worker i mod n_workers).

* ``solve_spectrum``        -- one process, one GPU;
* ``solve_spectrum_dist``   -- inside an initialised torch.distributed process
  group (one rank per GPU, e.g. under torchrun): each rank solves its
  wavelengths, one all-reduce (SUM of zero-padded arrays) gives every rank the
  full spectrum, the reported wall time is the maximum over the ranks;
* ``solve_spectrum_multi_gpu`` -- the reference's entry point: spawns one
  worker per GPU and runs ``solve_spectrum_dist`` in them.
"""
import os
import time

import numpy as np


def shard(n, rank, world):
    """Indices of the wavelengths rank ``rank`` of ``world`` solves (round robin)."""
    return list(range(rank, n, world))


def _make_solver(cp, pol, dirs, bem_class=None, **bem_kwargs):
    """solve_one(enei) -> (ext (npol,), sca (npol,)) with a GPU BEM solver."""
    from .planewave import PlaneWaveRet
    if bem_class in (None, "BEMRet"):
        from .bem import BEMRet as cls
    elif bem_class in ("BEMRetIter",):
        from .bem_iter import BEMRetIter as cls
    else:
        cls = bem_class
    bem = cls(cp, **bem_kwargs)
    exc = PlaneWaveRet(np.asarray(pol, dtype=float), np.asarray(dirs, dtype=float))

    def solve_one(enei):
        sig, _ = bem.solve(exc.potential(cp, float(enei)))
        ext = np.atleast_1d(exc.extinction(sig))
        sca = np.atleast_1d(exc.scattering(sig)[0])
        return ext, sca
    return solve_one


def solve_spectrum(cp, enei, pol, dirs, bem_class=None, **bem_kwargs):
    """Extinction / scattering spectra on one GPU: dict ext, sca (n_lambda x n_pol), enei, wall_s."""
    enei = np.asarray(enei, dtype=float)
    solve_one = _make_solver(cp, pol, dirs, bem_class, **bem_kwargs)
    t0 = time.time()
    rows = [solve_one(e) for e in enei]
    return {"ext": np.array([r[0] for r in rows]), "sca": np.array([r[1] for r in rows]), "enei": enei,
            "wall_s": time.time() - t0}


def sweep_dist(solve_one, enei, npol, device=None):
    """Shard ``enei`` over the ranks of the default process group, solve with
    ``solve_one`` and gather: returns (ext, sca, wall_max_s, my_indices).
    Every rank takes the same collective steps (one all-reduce for the
    results, one for the timing)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    n = len(enei)
    mine = shard(n, rank, world)
    buf = np.zeros((2, n, npol), dtype=np.float64)
    t0 = time.time()
    for i in mine:
        ext, sca = solve_one(enei[i])
        buf[0, i], buf[1, i] = ext, sca
    wall = time.time() - t0
    t = torch.as_tensor(buf, device=device)
    w = torch.tensor([wall], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        dist.all_reduce(w, op=dist.ReduceOp.MAX)
    out = t.cpu().numpy()
    return out[0], out[1], float(w.item()), mine


def solve_spectrum_dist(cp, enei, pol, dirs, bem_class=None, **bem_kwargs):
    """The sweep inside an initialised process group, one rank per GPU (device
    = LOCAL_RANK).  Returns the full spectrum on every rank."""
    import torch
    enei = np.asarray(enei, dtype=float)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    solve_one = _make_solver(cp, pol, dirs, bem_class, **bem_kwargs)
    npol = np.asarray(pol).reshape(-1, 3).shape[0]
    dev = torch.device("cuda", local) if torch.distributed.get_backend() == "nccl" else None
    ext, sca, wall, _ = sweep_dist(solve_one, enei, npol, device=dev)
    return {"ext": ext, "sca": sca, "enei": enei, "wall_s": wall}


def _worker(rank, world, port, particle_factory, enei, pol, dirs, bem_class, bem_kwargs, queue):
    import datetime
    import torch.distributed as dist
    os.environ["LOCAL_RANK"] = str(rank)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{}".format(port), rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=600))
    try:
        res = solve_spectrum_dist(particle_factory(), enei, pol, dirs, bem_class, **(bem_kwargs or {}))
        if rank == 0:
            queue.put(res)
    finally:
        dist.destroy_process_group()


def solve_spectrum_multi_gpu(particle_factory, enei, pol_dirs, prop_dirs, n_gpus=None, bem_kwargs=None,
                             bem_class=None, port=29533):
    """Reference-compatible entry point (mnpbem/utils/multi_gpu.py:148): one
    spawned worker per GPU, wavelength i on worker i mod n_gpus; returns dict
    ext, sca (n_lambda x n_pol), enei, wall_s (slowest worker)."""
    import torch
    import torch.multiprocessing as mp
    enei = np.asarray(enei, dtype=float)
    if n_gpus is None:
        n_gpus = torch.cuda.device_count()
    n_gpus = max(1, min(int(n_gpus), len(enei)))
    if n_gpus == 1:
        return solve_spectrum(particle_factory(), enei, pol_dirs, prop_dirs, bem_class, **(bem_kwargs or {}))
    ctx = mp.get_context("spawn")
    queue = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(n_gpus, port, particle_factory, enei, pol_dirs, prop_dirs, bem_class,
                                      bem_kwargs, queue), nprocs=n_gpus, join=True, start_method="spawn")
    return queue.get()
