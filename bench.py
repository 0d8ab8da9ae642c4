#!/usr/bin/env python
"""Throughput of the retarded BEM solve per wavelength on one B200 (or N replicas).

Workload: gold sphere dimer, 2 x trisphere(1444, 40 nm) = 5768 faces, 2 nm gap
on x, water (eps = 1.77), Drude gold (9.84, 9.0 eV, 0.067 eV), plane wave
polarised along x travelling along +z, wavelengths 650 + 0.05 s nm (step s).
A step is one full solve: Green assembly (G1, G2, H1, H2), Sigma / Delta build
with four LU factorisations, and the Eq. (19, 20) solve; with
--precision mixed the factors are complex64 (tcgen05 bf16x3 GEMMs) and the
solution is refined against the complex128 operator to max-residual 1e-12.
The one-time mesh precompute (refinement integrals) is excluded, as the metric
prescribes.

value : solves/s with the right-hand side resident on the device (CUDA events)
e2e   : solves/s through the public API, BEMRet.solve(exc.potential(p, enei)) +
        exc.extinction(sig): host excitation, host->device RHS copy, device->
        host copy of sig (events bracket host gaps too)
--impl reference : the CPU oracle (numpy/scipy restatement of the reference
        BEMRet path) on the host cores, same workload, same metric.

Multi-GPU: every rank solves its own wavelengths (replicas, weak scaling); the
time is the max over ranks; value = all ranks' solves / that time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s, 5768-face dimer: mixed+IR vs FP64 on 1 B200 at ext rel-err<=1e-8"
GOLD_EXT_650 = None  # filled from tests/golden/dimer_cfg1.npz
REF_MAX_SOLVES = 6   # timed CPU solves of the reference arm (each ~18 s)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--engine", default="bf16x3", choices=["bf16x3", "simt"])
    ap.add_argument("--fp64-steps", type=int, default=2, help="steps of the FP64 path timed for comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dimer(n=1444, diameter=40.0, gap=2.0):
    from mnpbem_b200 import ComParticle, EpsConst, EpsDrude, trisphere
    a, b = trisphere(n, diameter), trisphere(n, diameter)
    a.shift([-(diameter / 2 + gap / 2), 0, 0])
    b.shift([diameter / 2 + gap / 2, 0, 0])
    return ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")


POL = np.array([[1.0, 0.0, 0.0]])
DIR = np.array([[0.0, 0.0, 1.0]])


def wavelength(step, rank=0, world=1):
    return 650.0 + 0.05 * (step * world + rank)


def golden_ext():
    d = np.load(os.path.join(ROOT, "tests", "golden", "dimer_cfg1.npz"))
    return float(d["ext"])


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------- ours
def run_ours(args):
    import torch
    import torch.distributed as dist
    from mnpbem_b200 import PlaneWaveRet, _native
    from mnpbem_b200.bem import BEMRet

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    cp = dimer()
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp, precision=args.precision, engine=args.engine)  # mesh precompute (excluded)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def maxover(x):
        if world > 1:
            t = torch.tensor([x], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # device-resident right-hand sides for every step
    steps = args.warmup + args.steps
    rhs = []
    for s in range(steps):
        lam = wavelength(s, rank, world)
        b, npol = bem.rhs(exc.potential(cp, lam))
        rhs.append((lam, torch.as_tensor(b, dtype=torch.complex128, device=dev), npol))
    torch.cuda.synchronize()

    def device_step(lam, bt, npol):
        bem.clear()
        bem.init(lam)
        return bem.solve_device(bt, npol)

    for s in range(args.warmup):
        device_step(*rhs[s])
    torch.cuda.synchronize()
    L = _native.lib()
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    n0 = L.bem200_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    forms = set()
    irs = []
    e0.record()
    for s in range(args.warmup, steps):
        device_step(*rhs[s])
        irs.append(bem.last_ir)  # host values of the refinement (it synchronises once per sweep)
        forms.add(bem.last_pivoting)
    e1.record()
    torch.cuda.synchronize()
    launches = L.bem200_launch_count() - n0
    barrier()
    ck = clocks.stop()
    t_dev = maxover(e0.elapsed_time(e1) / 1e3)
    ir = bem.last_ir
    ir_max = maxover(max(r[1] for r in irs)) if irs and irs[0] else None
    if ir_max is not None and not ir_max <= bem.ir_tol:
        raise RuntimeError("bench: a timed step left the refinement residual at {:.3e} > ir_tol {:.1e}"
                           .format(ir_max, bem.ir_tol))

    # end to end through the public API (host excitation + transfers)
    barrier()
    torch.cuda.synchronize()
    h2d = d2h = 0
    exts = []
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    for s in range(args.warmup, steps):
        lam = wavelength(s, rank, world)
        bem.clear()
        sig, _ = bem.solve(exc.potential(cp, lam))
        exts.append(exc.extinction(sig))
        h2d += 16 * 8 * cp.n  # right-hand side (phi, a, alpha, De), complex128
        d2h += 16 * 8 * cp.n  # W1, W2 -> sig1, h1, sig2, h2
    e3.record()
    torch.cuda.synchronize()
    t_e2e = maxover(e2.elapsed_time(e3) / 1e3)

    # accuracy against the reference solver at 650 nm (complex128 oracle run)
    bem.clear()
    sig, _ = bem.solve(exc.potential(cp, 650.0))
    ext650 = exc.extinction(sig)
    gold = golden_ext()
    ext_err = abs(ext650 - gold) / abs(gold)

    # FP64 drop-in path on the same workload (comparison line)
    fp64_rate = None
    if args.precision == "mixed" and args.fp64_steps > 0:
        b64 = BEMRet(cp, precision="fp64")
        lam, bt, npol = rhs[0]
        b64.clear()
        b64.init(lam)
        b64.solve_device(bt, npol)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for s in range(args.fp64_steps):
            lam, bt, npol = rhs[args.warmup + s % args.steps]
            b64.clear()
            b64.init(lam)
            b64.solve_device(bt, npol)
        f1.record()
        torch.cuda.synchronize()
        fp64_rate = args.fp64_steps * world / maxover(f0.elapsed_time(f1) / 1e3)
        del b64
        torch.cuda.empty_cache()

    roof = roofline_gemm(dev) if rank == 0 else None
    fp64_tf = fp64_peak(dev) if (rank == 0 and fp64_rate) else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cp)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    value = args.steps * world / t_dev
    if forms == {"inverse"}:
        step_flops, step_note = 48.0, ("48 N^3 real flops: 4 complex inverses (8 N^3 each) and the 2 products "
                                       "Sigma_i = H_i G_i^-1 (8 N^3 each)")
    else:
        step_flops, step_note = 32.0, "32 N^3 real flops: 4 complex LUs, 2 N-RHS right solves, 1 inverse"
    out = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * t_dev / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64+c128" if args.precision == "mixed" else "c128",
        "data": "synthetic: seeded deterministic mesh (2 x trisphere(1444, 40 nm)), no dataset",
        "config": {
            "workload": "5768-face Au sphere dimer, 2 nm gap, water, Drude Au, x-pol +z, lambda = 650 + 0.05 s nm",
            "faces": cp.n,
            "precision": args.precision,
            "engine": args.engine if args.precision == "mixed" else "simt",
            "ir_iterations": ir[0] if ir else None,
            "ir_relres": ir[1] if ir else None,
            "ir_relres_max": ir_max,
            "ir_methods": sorted({r[2] for r in irs}) if irs and irs[0] else None,
            "factors": sorted(f for f in forms if f),
            "ext_650nm": ext650,
            "ext_rel_err_vs_reference_fp64": ext_err,
            "fp64_solves_per_s": round(fp64_rate, 4) if fp64_rate else None,
            "fp64_path_roofline": {
                "achieved_tflops": round(32.0 * cp.n ** 3 * fp64_rate / 1e12, 3),
                "peak_tflops": round(fp64_tf, 2),
                "peak_source": "cuBLAS DGEMM 4096^3 measured in this run (FP64 yardstick)",
                "frac": round(32.0 * cp.n ** 3 * fp64_rate / 1e12 / fp64_tf, 4),
            } if (fp64_rate and fp64_tf) else None,
            "mixed_over_fp64": round(value / fp64_rate, 3) if fp64_rate else None,
            "l2": "working set 2.1 GB of complex128 matrices per step (>> 126 MB L2); no flush needed",
            "parallelism": "replicas x{}".format(world),
        },
        "e2e": {"value": round(args.steps * world / t_e2e, 4), "unit": "solves/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": int(launches),
        "clocks": ck,
        "roofline": roof,
        "step_roofline": {
            "flops_per_step": step_flops * cp.n ** 3,
            "flops_note": step_note,
            "achieved_tflops": round(step_flops * cp.n ** 3 * args.steps / t_dev / 1e12, 2),  # per GPU
            "peak_tflops": roof["peak_sustained"] if roof else None,
            "frac": round(step_flops * cp.n ** 3 * args.steps / t_dev / 1e12 / roof["peak_sustained"], 4)
            if roof else None,
            "peak_source": roof["peak_sustained_source"] if roof else None,
        },
        "cpu_baseline": cpu,
    }
    print(json.dumps(out), flush=True)


def roofline_gemm(dev):
    """Dominant tensor-core kernel: complex64 bf16x3 GEMM of the Sigma / LU
    updates at the workload's top-level size (m = 5768, n = k = 2884), timed
    with CUDA events on its own stream.  achieved = 8 m n k algorithmic flops
    per launch / launch time; peak = measured dense bf16 (the tensor pipe runs 3
    bf16 products per complex64 product, so frac <= 1/3 by construction)."""
    import ctypes
    import torch
    from mnpbem_b200 import _native as nat
    m, n, k = 5768, 2884, 2884
    A = torch.randn(m, k, dtype=torch.complex64, device=dev)
    B = torch.randn(k, n, dtype=torch.complex64, device=dev)
    C = torch.zeros(m, n, dtype=torch.complex64, device=dev)
    wsb = int(nat.lib().bem200_gemm_workspace_size(1, m, n, k))
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    s = torch.cuda.current_stream()

    def go():
        nat.call("bem200_gemm", nat.C64, 1, m, n, k, one, nat.ptr(A), k, nat.ptr(B), n, zero, nat.ptr(C), n,
                 nat.ptr(ws), wsb, nat.stream_ptr(s))
    for _ in range(3):
        go()
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        go()
    e1.record(s)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    achieved = 8.0 * m * n * k / t / 1e12
    peak, src = 1590.0, "fallback (no MEASURED_PEAKS.json): earlier burst measurement on this pool"
    peak_s, src_s = 1400.0, "fallback (no MEASURED_PEAKS.json): sustained figure under the power cap on this pool"
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, src = float(mp["bf16_tflops"]), "measured bf16 burst"
        peak_s, src_s = float(mp["bf16_tflops_sustained"]), "measured bf16 sustained"
    except Exception:
        pass
    # DRAM bytes (read + write) of one launch of this GEMM from an ncu capture of the same shape
    # (profiles/gemm_bf16x3_5768x2884x2884.md): 1.251 GB read + 0.139 GB written
    traffic = 1.251e9 + 0.139e9
    return {"kernel": "tc::gemm_bf16x3_kernel (+ operand prep)", "bound": "tensor", "achieved": round(achieved, 2),
            "peak": peak, "peak_source": src, "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch",
            "algorithmic_flops_per_launch": 8.0 * m * n * k, "shape": [m, n, k], "ms_per_launch": round(1e3 * t, 3),
            "peak_sustained": peak_s, "peak_sustained_source": src_s}


def fp64_peak(dev):
    """FP64 yardstick of this GPU: cuBLAS DGEMM (torch.matmul, 4096^3) timed
    with CUDA events -- the denominator of the FP64 path's roofline fraction
    (the FP64 path runs its complex128 GEMMs on CUDA cores)."""
    import torch
    n = 4096
    A = torch.randn(n, n, dtype=torch.float64, device=dev)
    B = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(A, B)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        torch.matmul(A, B)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / 5
    return 2.0 * n ** 3 / t / 1e12


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(cp):
    """One per-wavelength solve of the CPU oracle (numpy/scipy complex128
    restatement of the reference path) on all host cores; the mesh precompute
    (refinement integrals) is excluded like in the GPU measurement."""
    from oracle.pipeline import OracleBEM
    ob = OracleBEM(cp)
    t0 = time.time()
    ob.solve(650.0, POL, DIR)
    t = time.time() - t0
    return {"value": round(1.0 / t, 5), "unit": "solves/s", "cores": os.cpu_count(), "cpu": cpu_model(), "kind": "port",
            "sample": "1 full solve (Green matrices + Sigma/Delta LU build + solve + ext/sca) of the 5768-face "
                      "dimer at 650 nm, {:.1f} s".format(t)}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pipeline import OracleBEM
    cp = dimer()
    ob = OracleBEM(cp)
    # one CPU solve takes ~18 s: one untimed warm-up and at most REF_MAX_SOLVES
    # timed solves keep the arm within a few minutes; the rate is per solve
    warm = min(args.warmup, 1)
    nsolve = max(1, min(args.steps, REF_MAX_SOLVES))
    for s in range(warm):
        ob.solve(wavelength(s), POL, DIR)
    t0 = time.time()
    for s in range(warm, warm + nsolve):
        ob.solve(wavelength(s), POL, DIR)
    t = time.time() - t0
    value = nsolve / t
    out = {
        "metric": METRIC, "value": round(value, 5), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic: seeded deterministic mesh (2 x trisphere(1444, 40 nm)), no dataset",
        "config": {"workload": "5768-face Au sphere dimer, 2 nm gap, water, Drude Au, x-pol +z, lambda = 650 + 0.05 s nm",
                   "faces": cp.n, "parallelism": "host cores"},
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 5), "unit": "solves/s", "cores": os.cpu_count(), "cpu": cpu_model(),
                         "kind": "port",
                         "sample": "{} timed full per-wavelength solves (after {} untimed) of the 5768-face dimer "
                                   "(CPU oracle, numpy/scipy complex128, all host threads)".format(nsolve, warm)},
        "e2e": {"value": round(value, 5), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
