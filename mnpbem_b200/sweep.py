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


def sweep_plan(sizes, nlambda, workers, schedule="interleave", units=None):
    """Per worker, the list of (mesh index, wavelength indices) it solves.
    ``units`` (mesh -> wavelength indices) restricts the plan to a share of
    the (mesh, wavelength) work; by default every mesh at every wavelength."""
    nm = len(sizes)
    if units is None:
        units = {m: np.arange(nlambda) for m in range(nm)}
    meshes = [m for m in range(nm) if len(units.get(m, ())) > 0]
    if schedule == "mesh":
        parts = lpt([float(sizes[m]) ** 3 for m in meshes], workers)
        return [[(meshes[i], np.asarray(units[meshes[i]])) for i in parts[w]] for w in range(workers)]
    if schedule != "interleave":
        raise ValueError("sweep_plan: schedule must be 'interleave' or 'mesh'")
    order = sorted(meshes, key=lambda m: -sizes[m])
    plan = []
    for w in range(workers):
        r = (w * len(order)) // workers
        items = [(m, np.asarray(units[m])[w::workers]) for m in order[r:] + order[:r]]
        plan.append([(m, lam) for m, lam in items if len(lam)])
    return plan


def partition_units(sizes, nlambda, world):
    """Longest processing time first over the (mesh, wavelength) units with
    cost n^3: for each rank, a dict mesh -> sorted wavelength indices."""
    units = [(m, i) for m in range(len(sizes)) for i in range(nlambda)]
    parts = lpt([float(sizes[m]) ** 3 for m, _ in units], world)
    out = []
    for p in parts:
        d = {}
        for u in p:
            m, i = units[u]
            d.setdefault(m, []).append(i)
        out.append({m: np.array(sorted(v)) for m, v in d.items()})
    return out


class _BEMSolver:
    """(mesh, wavelength) -> (ext, sca) with one resident BEMRet per mesh."""

    def __init__(self, particle, pol, dirs, precision, engine, **bem_kwargs):
        from .bem import BEMRet
        from .planewave import PlaneWaveRet
        self.bem = BEMRet(particle, precision=precision, engine=engine, **bem_kwargs)
        self.exc = PlaneWaveRet(pol, dirs)

    def prepare(self):
        self.bem._alloc()    # workspaces now, not inside the timed loops

    def __call__(self, enei):
        r = self.bem.cross_sections(self.exc, float(enei))
        return r["ext"], r["sca"]


def solve_sweep(particles, enei, pol, dirs, precision="mixed", workers=4, engine="bf16x3", schedule="interleave",
                units=None, solver_factory=None, **bem_kwargs):
    """Extinction and scattering of every particle at every wavelength (or of
    the (mesh, wavelength) ``units`` given, mesh -> wavelength indices; the
    others stay 0).

    Returns a dict: ext, sca ((nmesh, nlambda, npol) arrays), setup_s (solver
    construction for every (worker, mesh) pair: refinement tables,
    workspaces), sweep_s (the wavelength loops, all workers), solves (units x
    npol), solves_per_s (solves / sweep_s), per_worker seconds and the plan.
    ``solver_factory(particle, pol, dirs)`` may replace the GPU solver (an
    object called with a wavelength, returning (ext, sca))."""
    import torch
    enei = np.asarray(enei, dtype=float).ravel()
    pol = np.atleast_2d(np.asarray(pol, dtype=float))
    dirs = np.atleast_2d(np.asarray(dirs, dtype=float))
    npol = pol.shape[0]
    nm = len(particles)
    cuda = solver_factory is None
    if cuda:
        def solver_factory(p, pol_, dirs_):
            return _BEMSolver(p, pol_, dirs_, precision, engine, **bem_kwargs)
    workers = max(1, int(workers))
    if schedule == "mesh":
        workers = min(workers, nm)
    else:
        workers = min(workers, len(enei))
    plan = sweep_plan([p.n for p in particles], len(enei), workers, schedule, units)
    # the current device is per host thread: the workers adopt the caller's, on
    # which every BEMRet below allocates its workspaces
    dev = torch.cuda.current_device() if cuda else None
    t0 = time.perf_counter()
    solvers = [{m: solver_factory(particles[m], pol, dirs) for m, _ in plan[w]} for w in range(workers)]
    for per in solvers:
        for s_ in per.values():
            if hasattr(s_, "prepare"):
                s_.prepare()
    if cuda:
        torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    ext = np.zeros((nm, len(enei), npol))
    sca = np.zeros_like(ext)
    per_worker = [0.0] * workers
    errors = []
    start = threading.Barrier(workers + 1)

    def run(w):
        try:
            if cuda:
                torch.cuda.set_device(dev)
            stream = torch.cuda.Stream(device=dev) if cuda else None
            start.wait()
            tw = time.perf_counter()
            ctx = torch.cuda.stream(stream) if cuda else _nullcontext()
            with ctx:
                for m, lam in plan[w]:
                    for i in lam:
                        ext[m, i], sca[m, i] = solvers[w][m](enei[i])
                if cuda:
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
    if cuda:
        torch.cuda.synchronize()
    sweep = time.perf_counter() - t1
    if errors:
        raise errors[0]
    solves = sum(len(lam) for p in plan for _, lam in p) * npol
    return {"ext": ext, "sca": sca, "setup_s": setup, "sweep_s": sweep, "solves": solves,
            "solves_per_s": solves / sweep if sweep > 0 else float("inf"), "per_worker_s": per_worker,
            "plan": [[(int(m), len(lam)) for m, lam in p] for p in plan]}


def autotune_sweep(particles, enei, pol, dirs, candidates=((2, "interleave"), (4, "interleave"), (8, "interleave"),
                                                          (2, "mesh")), probe=4, **kw):
    """Pick the (workers, schedule) of ``solve_sweep`` for this batch by timing
    each candidate on ``probe`` wavelengths spread over the sweep (every mesh
    at each of them).  Returns (best candidate, {candidate: solves/s}).  The
    probe solves are real solves; their cost is a few wavelengths per
    candidate, against the whole sweep."""
    enei = np.asarray(enei, dtype=float).ravel()
    pick = np.unique(np.linspace(0, len(enei) - 1, max(1, min(probe, len(enei)))).round().astype(int))
    units = {m: pick for m in range(len(particles))}
    rates = {}
    for workers, schedule in candidates:
        r = solve_sweep(particles, enei, pol, dirs, workers=workers, schedule=schedule, units=units, **kw)
        rates[(workers, schedule)] = r["solves_per_s"]
    best = max(rates, key=rates.get)
    return best, rates


class _nullcontext:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def solve_sweep_dist(particles, enei, pol, dirs, device=None, **kw):
    """The uneven sweep inside an initialised process group, one rank per GPU:
    the (mesh, wavelength) units are split over the ranks by longest
    processing time first (cost n^3, ``partition_units``), every rank runs
    ``solve_sweep`` on its share, and two all-reduces (SUM of the zero-padded
    cross sections, MAX of the sweep time) give every rank the whole result.
    No other exchange: the units are independent.

    ``device`` holds the all-reduce buffers; by default the rank's GPU
    (LOCAL_RANK) when the backend is NCCL, else the CPU.  With a GPU solver
    the sweep runs on the current device, which is set to LOCAL_RANK when a
    CUDA device is available and the caller has not chosen one."""
    import os

    import torch
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if kw.get("solver_factory") is None and torch.cuda.is_available():
        torch.cuda.set_device(local % torch.cuda.device_count())
    if device is None and dist.is_initialized() and dist.get_backend() == "nccl":
        device = torch.device("cuda", local % torch.cuda.device_count())
    enei = np.asarray(enei, dtype=float).ravel()
    share = partition_units([p.n for p in particles], len(enei), world)[rank]
    r = solve_sweep(particles, enei, pol, dirs, units=share, **kw)
    buf = torch.as_tensor(np.stack([r["ext"], r["sca"]]), device=device)
    wall = torch.tensor([r["sweep_s"]], dtype=torch.float64, device=device)
    solves = torch.tensor([float(r["solves"])], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)
        dist.all_reduce(wall, op=dist.ReduceOp.MAX)
        dist.all_reduce(solves, op=dist.ReduceOp.SUM)
    out = buf.cpu().numpy()
    w = float(wall.item())
    n = int(solves.item())
    return {"ext": out[0], "sca": out[1], "sweep_s": w, "solves": n, "solves_per_s": n / w if w > 0 else float("inf"),
            "share": {int(m): v.tolist() for m, v in share.items()}}
