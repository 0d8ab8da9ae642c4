"""Single-stage timing and profiling cases of the retarded BEM solve.

    python -m mnpbem_b200.microbench step  [--faces 1444] [--precision mixed|fp64] [--steps 1] [--warmup 1]
    python -m mnpbem_b200.microbench green [--faces 1444] [--dtype c128|c64] [--reps 3]
    python -m mnpbem_b200.microbench gemm  [--m 5768 --n 2884 --k 2884] [--dtype c64] [--engine 1] [--reps 3]
    python -m mnpbem_b200.microbench getrf [--n 5768] [--dtype c64] [--engine 1] [--reps 1] [--tournament | --diagonal]
    python -m mnpbem_b200.microbench hmat  [--faces 1444] [--cleaf 200] [--htol 1e-6] [--reps 3]
    python -m mnpbem_b200.microbench iter  [--faces 1444] [--hmatrix] [--noprecond] [--tol 1e-10]
    python -m mnpbem_b200.microbench large [--side 3 | --shape cube] [--hmatrix] [--tol 1e-8]
    python -m mnpbem_b200.microbench sweep [--seed 0] [--nlambda 128] [--workers 4] [--schedule interleave|mesh]
    python -m mnpbem_b200.microbench shape [--nlambda 5] [--ndir 32] [--check 4] [--precision mixed]
    python -m mnpbem_b200.microbench peaks [--m 8192] [--reps 5]
    python -m mnpbem_b200.microbench vgrad [--shape rod|cube] [--nlambda 5] [--check 2] [--precision mixed]

``step`` runs whole per-wavelength solves (assembly + init + solve) of the
sphere dimer (two trisphere(faces) spheres, 2 nm gap, water, Drude gold,
x-polarised plane wave along +z); the other cases run one library entry point
on seeded inputs.  Each prints one JSON line with the CUDA-event time per
call.  These small cases are what the kernel profiles are taken on.
"""
import argparse
import ctypes
import json
import sys
import time

import numpy as np


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _timed(fn, reps):
    import torch
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def dimer(faces=1444, diameter=40.0, gap=2.0):
    from . import ComParticle, EpsConst, EpsDrude, trisphere
    a, b = trisphere(faces, diameter), trisphere(faces, diameter)
    a.shift([-(diameter / 2 + gap / 2), 0, 0])
    b.shift([diameter / 2 + gap / 2, 0, 0])
    return ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")


def case_step(a):
    import torch
    from . import PlaneWaveRet
    from .bem import BEMRet
    cp = dimer(a.faces)
    exc = PlaneWaveRet(np.array([[1.0, 0, 0]]), np.array([[0, 0, 1.0]]))
    bem = BEMRet(cp, precision=a.precision, engine=a.engine)
    b, npol = bem.rhs(exc.potential(cp, 650.0))
    bt = torch.as_tensor(b, dtype=torch.complex128, device="cuda")

    def one():
        bem.clear()
        bem.init(650.0)
        bem.solve_device(bt, npol)
    for _ in range(a.warmup):
        one()
    ms = _timed(one, a.steps)
    # one more step with the init's stage timer and events around assembly / init / solve
    bem._phase_buf = (ctypes.c_float * 4)()
    bem.clear()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed_step")  # lets a profiler select this step's kernels
    e[0].record()
    bem.init(650.0)
    e[1].record()
    bem.solve_device(bt, npol)
    e[2].record()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    bem._phase_buf = None
    ph = bem.last_init_phases_ms
    return {"case": "step", "faces": cp.n, "precision": a.precision, "ms_per_step": ms, "ir": bem.last_ir,
            "phases_ms": {"assembly_init_total": e[0].elapsed_time(e[1]), "solve_ir": e[1].elapsed_time(e[2]),
                          "lu_g1_g2_sigma1_sigma2": ph[0], "lu_delta": ph[1], "delta_inverse": ph[2],
                          "sigma_lu_sigma": ph[3]}}


def case_green(a):
    import torch
    from .greenfun import CompGreenRet
    cp = dimer(a.faces)
    g = CompGreenRet(cp, cp)
    n = cp.n
    dt = torch.complex128 if a.dtype == "c128" else torch.complex64
    out = [torch.empty((n, n), dtype=dt, device="cuda") for _ in range(4)]
    g.bem_matrices(650.0, dtype=a.dtype, out=out)
    ms = _timed(lambda: g.bem_matrices(650.0, dtype=a.dtype, out=out), a.reps)
    nbytes = 4 * n * n * (16 if a.dtype == "c128" else 8)
    return {"case": "green", "faces": n, "dtype": a.dtype, "ms": ms, "write_GBps": nbytes / ms / 1e6,
            "nref": g.refined.nref}


def case_gemm(a):
    import torch
    from . import _native as nat
    m, n, k = a.m, a.n, a.k
    dt = torch.complex128 if a.dtype == "c128" else torch.complex64
    code = nat.C128 if a.dtype == "c128" else nat.C64
    gen = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(m, k, dtype=dt, device="cuda", generator=gen)
    B = torch.randn(k, n, dtype=dt, device="cuda", generator=gen)
    C = torch.zeros(m, n, dtype=dt, device="cuda")
    wsb = int(nat.lib().bem200_gemm_workspace_size(a.engine, m, n, k))
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)

    def go():
        nat.call("bem200_gemm", code, a.engine, m, n, k, one, nat.ptr(A), k, nat.ptr(B), n, zero, nat.ptr(C), n,
                 nat.ptr(ws), wsb, nat.stream_ptr())
    go()
    ms = _timed(go, a.reps)
    return {"case": "gemm", "m": m, "n": n, "k": k, "dtype": a.dtype, "engine": a.engine, "ms": ms,
            "complex_TFLOPs": 8.0 * m * n * k / ms / 1e9,
            "operand_GBs": A.element_size() * (m * k + k * n + 2 * m * n) / ms / 1e6}


def case_getrf(a):
    import torch
    from . import _native as nat
    n = a.n
    dt = torch.complex128 if a.dtype == "c128" else torch.complex64
    code = nat.C128 if a.dtype == "c128" else nat.C64
    gen = torch.Generator(device="cuda").manual_seed(0)
    A0 = torch.randn(n, n, dtype=dt, device="cuda", generator=gen)
    if a.diagonal:  # a column-dominant diagonal, as the BEM factor matrices have: no row exchanges
        A0 += 100.0 * torch.eye(n, dtype=dt, device="cuda")
    A = torch.empty_like(A0)
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = int(nat.lib().bem200_getrf_workspace_size(code, a.engine, n))
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")

    flags = 2 if a.tournament else (4 if a.diagonal else 0)

    def go():
        A.copy_(A0)
        nat.call("bem200_getrf_ex", code, a.engine, n, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
                 nat.ptr(ws), wsb, flags, a.la_nb, nat.stream_ptr())
    go()
    # backward error of a solve with these factors: |A0 x - b| / (|A0| |x|)
    b = torch.randn(n, 2, dtype=dt, device="cuda", generator=gen)
    x = b.clone()
    scr = torch.empty(int(nat.lib().bem200_getrs_workspace_size(code, n, 2)), dtype=torch.uint8, device="cuda")
    nat.call("bem200_getrs", code, 0, n, 2, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(x), 2, None, 0, nat.ptr(scr),
             None, nat.stream_ptr())
    A64, x64 = A0.to(torch.complex128), x.to(torch.complex128)
    berr = float(torch.linalg.matrix_norm(A64 @ x64 - b.to(torch.complex128), ord=float("inf"))
                 / (torch.linalg.matrix_norm(A64, ord=float("inf")) * torch.linalg.matrix_norm(x64, ord=float("inf"))))
    if a.graph:
        # the same factorisation replayed from a CUDA graph (no host launch work)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            go()
        g.replay()
        ms = _timed(g.replay, a.reps)
    else:
        ms = _timed(go, a.reps)
    return {"case": "getrf", "n": n, "dtype": a.dtype, "engine": a.engine, "graph": bool(a.graph),
            "pivoting": "tournament (complex64 panels > 512 rows)" if a.tournament else (
                "diagonal (checked, no row exchanges)" if a.diagonal else "partial"), "ms": ms,
            "TFLOPs": 8.0 / 3.0 * n ** 3 / ms / 1e9, "info": int(info.item()), "backward_error": berr}


def case_inverse(a):
    """bem200_inverse_nopiv on a column-dominant random matrix (no row
    exchanges needed, as the BEM factor matrices)."""
    import torch
    from . import _native as nat
    n = a.n
    dt = torch.complex128 if a.dtype == "c128" else torch.complex64
    code = nat.C128 if a.dtype == "c128" else nat.C64
    gen = torch.Generator(device="cuda").manual_seed(0)
    A0 = torch.randn(n, n, dtype=dt, device="cuda", generator=gen) + 4.0 * n ** 0.5 * torch.eye(n, dtype=dt,
                                                                                               device="cuda")
    A = torch.empty_like(A0)
    L = nat.lib()
    scr = torch.empty(int(L.bem200_inverse_nopiv_workspace_size(code, n)), dtype=torch.uint8, device="cuda")
    wsb = int(L.bem200_gemm_workspace_size(a.engine, n, n, n // 2 + 64)) if a.engine else 0
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")

    def go():
        A.copy_(A0)
        nat.call("bem200_inverse_nopiv", code, a.engine, n, nat.ptr(A), n, nat.ptr(ws), wsb, nat.ptr(scr), 1e-2,
                 nat.ptr(info), nat.stream_ptr())
    go()
    if a.graph:
        # the same inversion replayed from a CUDA graph (no host launch work)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            go()
        g.replay()
        ms = _timed(g.replay, a.reps)
    else:
        ms = _timed(go, a.reps)
    res = float((A.to(torch.complex128) @ A0.to(torch.complex128)
                 - torch.eye(n, dtype=torch.complex128, device="cuda")).abs().max())
    return {"case": "inverse", "n": n, "dtype": a.dtype, "engine": a.engine, "graph": bool(a.graph), "ms": ms,
            "TFLOPs": 8.0 * n ** 3 / ms / 1e9, "info": int(info.item()), "max|A^-1 A - I|": res}


def case_hmat(a):
    """H-matrix of the dimer's G1: build of the four BEM matrices (--fill green:
    dense leaves and ACA rows / columns computed on demand; dense: dense
    assembly, then ACA), compression and the matvec with 8 right-hand columns."""
    import torch
    from .greenfun import CompGreenRet
    from .hmatrix import BEMHMatrices
    cp = dimer(a.faces)
    g = CompGreenRet(cp, cp)
    hb = BEMHMatrices(cp, g, htol=a.htol, kmax=100, cleaf=a.cleaf, eta=2.5)
    fill = "green" if a.fill == "auto" else a.fill
    hb.build(650.0, fill=fill)
    ms_build = _timed(lambda: hb.build(650.0, fill=fill), 1)
    h = hb.H[0]
    n, w = cp.n, 8
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(n, w, dtype=torch.complex128, device="cuda", generator=gen)
    y = torch.empty_like(x)
    h.matvec(x, y, w)
    ms_mv = _timed(lambda: h.matvec(x, y, w), a.reps)
    stored = int(h._doff_h[-1]) + int(np.sum(h.ranks.astype(np.int64) * (h._lb[:, 1] + h._lb[:, 3])))
    nbytes = 16 * stored
    return {"case": "hmat", "faces": n, "cleaf": a.cleaf, "htol": a.htol, "fill": fill,
            "ms_build_4_matrices": ms_build,
            "compression": hb.compression(), "dense_blocks": h.ndense, "lowrank_blocks": h.nlow,
            "max_rank": int(h.ranks.max()) if h.nlow else 0, "ms_matvec_w8": ms_mv,
            "matvec_factor_GBps": nbytes / ms_mv / 1e6, "dense_matvec_bytes": 16 * n * n}


def case_iter(a):
    """BEMRetIter solves of the dimer (dense or H-matrix operator, complex64
    factors as preconditioner): init (+ compression) and GMRES per wavelength."""
    import torch
    from . import PlaneWaveRet
    from .bem_iter import BEMRetIter
    cp = dimer(a.faces)
    exc = PlaneWaveRet(np.array([[1.0, 0, 0]]), np.array([[0, 0, 1.0]]))
    bem = BEMRetIter(cp, hmatrix=a.hmatrix, cleaf=a.cleaf, htol=a.htol, tol=a.tol,
                     precond=None if a.noprecond else "hmat")
    out = {"case": "iter", "faces": cp.n, "hmatrix": a.hmatrix, "tol": a.tol, "precond": not a.noprecond}
    for rep in range(2):
        lam = 650.0 + rep
        e0, e1, e2 = _events() + (torch.cuda.Event(enable_timing=True),)
        torch.cuda.synchronize()
        e0.record()
        bem.init(lam)
        e1.record()
        b, npol = bem._bem.rhs(exc.potential(cp, lam))
        bt = torch.as_tensor(b, dtype=torch.complex128, device="cuda")
        bem.solve_device(bt, npol)
        e2.record()
        torch.cuda.synchronize()
        out["ms_init"], out["ms_solve"] = e0.elapsed_time(e1), e1.elapsed_time(e2)
    out["iters"], out["relres"] = bem.last.iter, bem.last.relres
    return out


def sphere_array(side=3, faces=1444, diameter=40.0, gap=2.0, eps_b=1.0):
    """side x side gold spheres (trisphere(faces, diameter)) on a square grid in
    the xy plane with surface gaps ``gap``: 2884 side^2 faces at faces=1444."""
    from . import ComParticle, EpsConst, EpsDrude, trisphere
    parts = []
    pitch = diameter + gap
    for i in range(side):
        for j in range(side):
            q = trisphere(faces, diameter)
            q.shift([(i - (side - 1) / 2) * pitch, (j - (side - 1) / 2) * pitch, 0.0])
            parts.append(q)
    k = len(parts)
    return ComParticle([EpsConst(eps_b), EpsDrude(9.84, 9.0, 0.067)], parts, [[2, 1]] * k, *range(1, k + 1),
                       interp="curv")


def case_large(a):
    """One large solve (3 x 3 gold spheres, 25956 faces, or with --shape cube
    the rounded gold cube tricube(66, 100 nm, e = 0.25), 25344 curved quads;
    vacuum, 700 nm, x-pol): BEMRetIter with the complex64 tensor-core LU as
    preconditioner and the FP64 dense (or H-matrix) operator."""
    import torch
    from . import PlaneWaveRet
    from .bem_iter import BEMRetIter
    if a.shape == "cube":
        from . import ComParticle, EpsConst, EpsDrude
        from .geometry import tricube
        cp = ComParticle([EpsConst(1.0), EpsDrude(9.84, 9.0, 0.067)], [tricube(a.cube_n, 100.0, a.cube_e,
                                                                                 interp="curv")],
                         [[2, 1]], 1, interp="curv")
    else:
        cp = sphere_array(a.side)
    exc = PlaneWaveRet(np.array([[1.0, 0, 0]]), np.array([[0, 0, 1.0]]))
    e0, e1, e2 = _events() + (torch.cuda.Event(enable_timing=True),)
    torch.cuda.synchronize()
    e0.record()
    bem = BEMRetIter(cp, hmatrix=a.hmatrix, cleaf=a.cleaf, htol=a.htol, tol=a.tol, hmat_fill=a.fill,
                     precond=None if a.noprecond else "hmat", maxit=1000)
    bem.init(700.0)
    e1.record()
    sig, _ = bem.solve(exc.potential(cp, 700.0))
    e2.record()
    torch.cuda.synchronize()
    out = {"case": "large", "shape": a.shape, "faces": cp.n, "hmatrix": a.hmatrix, "fill": a.fill,
           "precond": not a.noprecond, "tol": a.tol, "ext": exc.extinction(sig),
           "sca": exc.scattering(sig)[0], "iters": bem.last.iter, "relres": bem.last.relres,
           "ms_ctor_init": e0.elapsed_time(e1), "ms_solve": e1.elapsed_time(e2),
           "max_mem_GB": torch.cuda.max_memory_allocated() / 1e9}
    if a.hmatrix:
        out["compression"] = bem._hmat.compression()
    return out


def case_sweep(a):
    """The uneven batch: 8 seeded spheres / ellipsoids / rods of 284 ... 5768
    faces (gold or silver, vacuum), nlambda wavelengths 450-900 nm, x and y
    polarisations along +z, complex64 factors + FP64 refinement, the (mesh,
    wavelength) work spread over ``workers`` streams.  ``check`` wavelengths per mesh are re-solved with
    the fp64 path and the largest extinction error is reported."""
    import torch
    from .bem import BEMRet
    from .planewave import PlaneWaveRet
    from .sweep import solve_sweep, uneven_meshes
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    enei = np.linspace(450.0, 900.0, a.nlambda)
    t0 = time.perf_counter()
    meshes = uneven_meshes(a.seed)
    mesh_s = time.perf_counter() - t0
    r = solve_sweep([m["p"] for m in meshes], enei, pol, dirs, precision=a.precision, workers=a.workers,
                    schedule=a.schedule)
    worst = 0.0
    rng = np.random.default_rng(a.seed + 1)
    exc = PlaneWaveRet(pol, dirs)
    for mi, m in enumerate(meshes):
        ref = BEMRet(m["p"])
        for i in rng.choice(len(enei), size=min(a.check, len(enei)), replace=False):
            e64 = ref.cross_sections(exc, float(enei[i]))["ext"]
            worst = max(worst, float(np.max(np.abs(r["ext"][mi, i] - e64) / np.abs(e64))))
        del ref
    torch.cuda.synchronize()
    return {"case": "sweep", "seed": a.seed, "faces": [m["n"] for m in meshes],
            "shapes": [m["shape"] for m in meshes], "metals": [m["metal"] for m in meshes],
            "nlambda": a.nlambda, "npol": 2, "workers": a.workers, "schedule": a.schedule,
            "precision": a.precision,
            "solves": r["solves"], "sweep_s": r["sweep_s"], "solves_per_s": r["solves_per_s"],
            "setup_s": r["setup_s"], "mesh_build_s": mesh_s,
            "e2e_solves_per_s": r["solves"] / (r["sweep_s"] + r["setup_s"] + mesh_s),
            "per_worker_s": [round(v, 3) for v in r["per_worker_s"]], "max_ext_relerr_vs_fp64": worst,
            "max_mem_GB": torch.cuda.max_memory_allocated() / 1e9}


def case_shape(a):
    """Gradients of the extinction of the gold rod trirod(20, 80, [41, 16, 31])
    (2400 curved faces, eps_b 1.77, x-pol along +z) at nlambda wavelengths
    600-800 nm: 32 seeded vertex directions (ShapeSensitivity) and the
    permittivity gradient; ``check`` directions at the middle wavelength are
    compared with central differences of full fp64 solves (step 1e-4 nm)."""
    import torch
    from . import BEMRet, ComParticle, EpsConst, EpsDrude, PlaneWaveRet
    from .adjoint import extinction_eps_gradient
    from .geometry import trirod
    from .shape import ShapeSensitivity, perturbed, random_directions
    cp = ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)], [trirod(20.0, 80.0, [41, 16, 31],
                                                                             interp="curv")],
                     [[2, 1]], 1, interp="curv")
    exc = PlaneWaveRet(np.array([[1.0, 0, 0]]), np.array([[0, 0, 1.0]]))
    D = random_directions(cp, a.ndir, seed=a.seed)
    enei = np.linspace(600.0, 800.0, a.nlambda)
    bem = BEMRet(cp, precision=a.precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sens = ShapeSensitivity(bem, D, 1e-4)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    exts, dexts, t_lam, t_eps = [], [], [], []
    for e in enei:
        t1 = time.perf_counter()
        ext, dext = sens.extinction(exc, float(e))
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        _, geps = extinction_eps_gradient(bem, exc, float(e), 2)
        torch.cuda.synchronize()
        t_lam.append(t2 - t1)
        t_eps.append(time.perf_counter() - t2)
        exts.append(float(ext[0]))
        dexts.append(dext[:, 0])
    mid = len(enei) // 2
    worst = 0.0
    for k in range(min(a.check, a.ndir)):
        e2 = []
        for s in (1.0, -1.0):
            q = perturbed(cp, s * 1e-4 * D[k])
            sig, _ = BEMRet(q).solve(exc.potential(q, float(enei[mid])))
            e2.append(float(exc.extinction(sig)))
        fd = (e2[0] - e2[1]) / 2e-4
        worst = max(worst, abs(dexts[mid][k] - fd) / np.max(np.abs(dexts[mid])))
    return {"case": "shape", "faces": cp.n, "nvert": int(D.shape[1]), "ndir": a.ndir, "nlambda": a.nlambda,
            "precision": a.precision, "ext": exts, "setup_s": t_setup, "s_per_lambda_32dir": t_lam,
            "s_per_lambda_eps_grad": t_eps, "max_fd_relerr": worst, "fd_checked": min(a.check, a.ndir),
            "max_mem_GB": torch.cuda.max_memory_allocated() / 1e9}


def case_vgrad(a):
    """Reverse-mode gradient of the extinction over every vertex coordinate
    (one transposed solve with the wavelength's factors, the operator
    derivative contracted on the GPU): the gold rod trirod(20, 80, [41, 16,
    31]) (2400 curved faces, eps_b 1.77) at nlambda wavelengths 600-800 nm,
    or with --shape cube the rounded gold cube tricube(66, 100 nm, e = 0.25)
    (25344 curved quads, vacuum) at 700 nm.  ``check`` seeded directions at
    the first wavelength are compared with central differences of full fp64
    solves (step 1e-4 nm)."""
    import torch
    from . import BEMRet, ComParticle, EpsConst, EpsDrude, PlaneWaveRet
    from .geometry import tricube, trirod
    from .shape import extinction_vertex_vjp, perturbed, random_directions
    if a.shape == "cube":
        cp = ComParticle([EpsConst(1.0), EpsDrude(9.84, 9.0, 0.067)],
                         [tricube(a.cube_n, 100.0, a.cube_e, interp="curv")], [[2, 1]], 1, interp="curv")
        enei = np.array([700.0])
    else:
        cp = ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)],
                         [trirod(20.0, 80.0, [41, 16, 31], interp="curv")], [[2, 1]], 1, interp="curv")
        enei = np.linspace(600.0, 800.0, a.nlambda)
    exc = PlaneWaveRet(np.array([[1.0, 0, 0]]), np.array([[0, 0, 1.0]]))
    bem = BEMRet(cp, precision=a.precision)
    t_init, t_grad, exts, grads = [], [], [], []
    for e in enei:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bem.init(float(e))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ext, g = extinction_vertex_vjp(bem, exc, float(e))
        torch.cuda.synchronize()
        t_init.append(t1 - t0)
        t_grad.append(time.perf_counter() - t1)
        exts.append(float(ext[0]))
        grads.append(g)
    worst = 0.0
    D = random_directions(cp, max(a.check, 1), seed=a.seed)
    for k in range(a.check):
        e2 = []
        for s in (1.0, -1.0):
            q = perturbed(cp, s * 1e-4 * D[k])
            e2.append(float(BEMRet(q).cross_sections(exc, float(enei[0]))["ext"][0]))
        fd = (e2[0] - e2[1]) / 2e-4
        got = float(np.sum(grads[0] * D[k]))
        worst = max(worst, abs(got - fd) / max(abs(fd), 1e-12))
    return {"case": "vgrad", "shape": a.shape, "faces": cp.n, "nvert": int(grads[0].shape[0]),
            "precision": a.precision, "enei": enei.tolist(), "ext": exts, "s_init_per_lambda": t_init,
            "s_solve_adjoint_gradient_per_lambda": t_grad, "fd_checked": a.check, "max_fd_relerr": worst,
            "max_mem_GB": torch.cuda.max_memory_allocated() / 1e9}


def case_peaks(a):
    """Reference pipe rates of this GPU, from cuBLAS through torch.matmul
    (library GEMMs used only as a yardstick): FP64 (DGEMM, ZGEMM), FP32
    without and with TF32, and dense bf16; m = n = k = a.m (default 8192),
    CUDA events over a.reps launches after one warm-up.  Complex GEMMs count
    8 real flops per multiply-add."""
    import torch
    n = a.m if a.m != 5768 else 8192
    out = {"case": "peaks", "size": n}
    prev = torch.backends.cuda.matmul.allow_tf32
    try:
        for name, dt, tf32, cx in (("fp64", torch.float64, False, False), ("c128", torch.complex128, False, True),
                                   ("fp32", torch.float32, False, False), ("tf32", torch.float32, True, False),
                                   ("bf16", torch.bfloat16, False, False)):
            torch.backends.cuda.matmul.allow_tf32 = tf32
            m = n // 2 if cx else n
            A = torch.randn(m, m, dtype=dt, device="cuda")
            B = torch.randn(m, m, dtype=dt, device="cuda")
            torch.matmul(A, B)
            ms = _timed(lambda: torch.matmul(A, B), a.reps)
            flops = (8.0 if cx else 2.0) * m ** 3
            out[name + "_tflops"] = round(flops / ms / 1e9, 2)
            del A, B
            torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["step", "green", "gemm", "getrf", "inverse", "hmat", "iter", "large", "sweep",
                                           "shape", "peaks", "vgrad"])
    ap.add_argument("--faces", type=int, default=1444)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--engine", type=int, default=1)
    ap.add_argument("--dtype", default="c128", choices=["c128", "c64"])
    ap.add_argument("--m", type=int, default=5768)
    ap.add_argument("--n", type=int, default=2884)
    ap.add_argument("--k", type=int, default=2884)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--graph", action="store_true", help="getrf: replay from a CUDA graph")
    ap.add_argument("--tournament", action="store_true", help="getrf: tournament pivoting of complex64 panels")
    ap.add_argument("--diagonal", action="store_true",
                    help="getrf: checked diagonal pivots (no pivot search) on a column-dominant matrix")
    ap.add_argument("--la-nb", dest="la_nb", type=int, default=0, help="getrf: look-ahead block width (0 = 128)")
    ap.add_argument("--cleaf", type=int, default=200)
    ap.add_argument("--htol", type=float, default=1e-6)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--hmatrix", action="store_true")
    ap.add_argument("--noprecond", action="store_true")
    ap.add_argument("--side", type=int, default=3)
    ap.add_argument("--shape", default="spheres", choices=["spheres", "cube", "rod"])
    ap.add_argument("--cube-n", dest="cube_n", type=int, default=66)
    ap.add_argument("--cube-e", dest="cube_e", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--nlambda", type=int, default=128)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--schedule", default="interleave", choices=["interleave", "mesh"])
    ap.add_argument("--check", type=int, default=1)
    ap.add_argument("--ndir", type=int, default=32)
    ap.add_argument("--fill", default="auto", choices=["auto", "green", "dense"])
    a = ap.parse_args(argv)
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("microbench needs a CUDA device")
    if a.case == "step":
        a.engine = {0: "simt", 1: "bf16x3"}[a.engine]
    out = {"step": case_step, "green": case_green, "gemm": case_gemm, "getrf": case_getrf, "inverse": case_inverse,
           "hmat": case_hmat,
           "iter": case_iter, "large": case_large, "sweep": case_sweep,
           "shape": case_shape, "peaks": case_peaks, "vgrad": case_vgrad}[a.case](a)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
