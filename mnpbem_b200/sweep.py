"""Wavelength sweeps over many meshes of uneven size on one GPU.

The reference solves such a batch as a loop: one BEMRet per mesh, one
``bem.solve(exc.potential(p, enei))`` per wavelength (its production
parallel axis, mnpbem/utils/multi_gpu.py:148-260, only spreads that loop over
GPUs).  Here every mesh keeps its own BEMRet (workspaces, refinement tables
and FP64 operator resident in HBM for the whole sweep) and the (mesh,
wavelength) work is spread over a few host worker threads, each issuing its
share on its own CUDA stream.  A large mesh keeps the tensor cores busy with its
LU updates while the panels and triangular sweeps of another mesh, which cannot
fill 148 SMs alone, run beside it.  Two schedules:

* ``interleave`` (default): worker w takes the wavelengths i = w (mod W) of
  every mesh, starting from a different mesh (the meshes sorted by size and
  rotated by w nmesh / W), so each worker has the same load and large and small
  meshes overlap.  Each worker keeps its own BEMRet per mesh.
* ``mesh``: whole meshes go to workers by longest processing time first, with
  n^3 as the cost.

Every per-wavelength step stays on the GPU (right-hand side, factors, solve
with FP64 refinement, far fields); only the (npol,) cross sections return.

``uneven_meshes(seed)`` builds a seeded batch of uneven meshes with the reference's
generators: spheres (trisphere, curved), ellipsoids (triellipsoid, flat) and
capped rods (trirod, curved) with face counts 284 ... 5768, seeded sizes and
gold or silver Drude metals.
"""
import threading
import time

import numpy as np

from .geometry import ComParticle, triellipsoid, trirod, trisphere
from .materials import EpsConst, EpsDrude

GOLD = (9.84, 9.0, 0.067)      # eps_inf, hbar w_p (eV), hbar gamma (eV)
SILVER = (3.7, 9.17, 0.021)

# face count -> (shape, resolution); rods: n = [nphi, ntheta, nz] gives
# (nphi - 1) (2 (ntheta - 1) + nz - 1) faces, ellipsoids 2 nverts - 4,
# trisphere(n) 2 n - 4
UNEVEN_SHAPES = (
    (284, "sphere", 144),
    (760, "ellipsoid", 382),
    (1296, "rod", (25, 14, 29)),
    (2000, "ellipsoid", 1002),
    (2884, "sphere", 1444),
    (3600, "rod", (41, 21, 51)),
    (4800, "ellipsoid", 2402),
    (5768, "rod", (57, 31, 44)),
)


def uneven_meshes(seed=0, eps_b=1.0, shapes=UNEVEN_SHAPES):
    """Seeded particles of uneven size: a list of dicts with the ComParticle
    ('p'), its face count, shape, dimensions (nm) and metal.  Draws
    (numpy default_rng(seed)): sphere diameter 2 U[10, 40], ellipsoid semi-axes
    U[10, 40], rod radius U[8, 20] and length U[max(40, 2 r + 10), 120],
    metal gold or silver with equal odds."""
    rng = np.random.default_rng(seed)
    out = []
    for nf, shape, res in shapes:
        metal = "gold" if rng.random() < 0.5 else "silver"
        if shape == "sphere":
            dims = {"diameter": 2 * rng.uniform(10, 40)}
            part = trisphere(res, dims["diameter"])
            interp = "curv"
        elif shape == "ellipsoid":
            dims = {"axes": rng.uniform(10, 40, size=3)}
            part = triellipsoid(res, dims["axes"])
            interp = "flat"
        else:
            r = rng.uniform(8, 20)
            dims = {"diameter": 2 * r, "length": rng.uniform(max(40.0, 2 * r + 10), 120)}
            part = trirod(dims["diameter"], dims["length"], list(res), interp="curv")
            interp = "curv"
        drude = GOLD if metal == "gold" else SILVER
        cp = ComParticle([EpsConst(eps_b), EpsDrude(*drude)], [part], [[2, 1]], 1, interp=interp)
        if cp.n != nf:
            raise RuntimeError("uneven_meshes: {} gave {} faces, expected {}".format(shape, cp.n, nf))
        out.append({"p": cp, "n": cp.n, "shape": shape, "dims": dims, "metal": metal})
    return out


def lpt(costs, workers):
    """Longest processing time first: lists of item indices per worker."""
    load = [0.0] * workers
    parts = [[] for _ in range(workers)]
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        w = int(np.argmin(load))
        parts[w].append(i)
        load[w] += costs[i]
    return parts


def sweep_plan(sizes, nlambda, workers, schedule="interleave"):
    """Per worker, the list of (mesh index, wavelength indices) it solves."""
    nm = len(sizes)
    if schedule == "mesh":
        parts = lpt([float(n) ** 3 for n in sizes], workers)
        return [[(m, np.arange(nlambda)) for m in parts[w]] for w in range(workers)]
    if schedule != "interleave":
        raise ValueError("sweep_plan: schedule must be 'interleave' or 'mesh'")
    order = sorted(range(nm), key=lambda m: -sizes[m])
    plan = []
    for w in range(workers):
        r = (w * nm) // workers
        plan.append([(m, np.arange(w, nlambda, workers)) for m in order[r:] + order[:r]])
    return plan


def solve_sweep(particles, enei, pol, dirs, precision="mixed", workers=4, engine="bf16x3", schedule="interleave",
                **bem_kwargs):
    """Extinction and scattering of every particle at every wavelength.

    Returns a dict: ext, sca ((nmesh, nlambda, npol) arrays), setup_s (BEMRet
    construction for every (worker, mesh) pair: refinement tables,
    workspaces), sweep_s (the wavelength loops, all workers), solves
    (nmesh * nlambda * npol), solves_per_s (solves / sweep_s), per_worker
    seconds and the plan."""
    import torch
    from .bem import BEMRet
    from .planewave import PlaneWaveRet
    enei = np.asarray(enei, dtype=float).ravel()
    pol = np.atleast_2d(np.asarray(pol, dtype=float))
    dirs = np.atleast_2d(np.asarray(dirs, dtype=float))
    npol = pol.shape[0]
    nm = len(particles)
    workers = max(1, int(workers))
    if schedule == "mesh":
        workers = min(workers, nm)
    else:
        workers = min(workers, len(enei))
    plan = sweep_plan([p.n for p in particles], len(enei), workers, schedule)
    t0 = time.perf_counter()
    bems = [{m: BEMRet(particles[m], precision=precision, engine=engine, **bem_kwargs) for m, _ in plan[w]}
            for w in range(workers)]
    for per in bems:
        for b in per.values():
            b._alloc()    # workspaces now, not inside the timed loops
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    ext = np.zeros((nm, len(enei), npol))
    sca = np.zeros_like(ext)
    per_worker = [0.0] * workers
    errors = []
    start = threading.Barrier(workers + 1)

    def run(w):
        try:
            stream = torch.cuda.Stream()
            exc = PlaneWaveRet(pol, dirs)
            start.wait()
            tw = time.perf_counter()
            with torch.cuda.stream(stream):
                for m, lam in plan[w]:
                    for i in lam:
                        r = bems[w][m].cross_sections(exc, float(enei[i]))
                        ext[m, i], sca[m, i] = r["ext"], r["sca"]
                stream.synchronize()
            per_worker[w] = time.perf_counter() - tw
        except BaseException as exc_:  # reported on the calling thread
            errors.append(exc_)
            if not start.broken:
                start.abort()

    threads = [threading.Thread(target=run, args=(w,)) for w in range(workers)]
    for t in threads:
        t.start()
    try:
        start.wait()
    except threading.BrokenBarrierError:
        pass
    t1 = time.perf_counter()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    sweep = time.perf_counter() - t1
    if errors:
        raise errors[0]
    solves = nm * len(enei) * npol
    return {"ext": ext, "sca": sca, "setup_s": setup, "sweep_s": sweep, "solves": solves,
            "solves_per_s": solves / sweep, "per_worker_s": per_worker,
            "plan": [[(int(m), len(lam)) for m, lam in p] for p in plan]}
