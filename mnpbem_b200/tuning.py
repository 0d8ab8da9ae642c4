"""Autotuner of the LU tiling.

The dense LU (``bem200_getrf_ex`` / ``bem200_bem_init_ex``) factors block
columns of a look-ahead width nb: the panels and the next block column run on
a high-priority stream while the wide update of the rest runs beside them.  A
small nb shortens the critical path of each step but issues more, smaller
tensor-core GEMMs; a large nb the opposite.  The best width depends on n and on
the GPU, so it is measured: ``tune_lookahead`` times the factorisation of a
seeded random matrix of the same size and precision for each candidate width
(CUDA events) and keeps the fastest.  Results are cached per (device, dtype,
engine, n rounded to 256) in a JSON file (``BEM200_TUNE_CACHE``, default
``~/.cache/mnpbem_b200/lu_tiles.json``), so a sweep pays the probe once per mesh
size.
"""
import json
import os
import threading

from . import _native as nat

CANDIDATES = (64, 96, 128, 192, 256)
_LOCK = threading.Lock()
_MEM = {}


def _cache_path():
    return os.environ.get("BEM200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mnpbem_b200", "lu_tiles.json"))


def _load():
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(key, value):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load()
        data[key] = value
        tmp = path + ".tmp{}".format(os.getpid())
        with open(tmp, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: keep the result in memory only


def _key(dtype, engine, n):
    import torch
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    return "{}|{}|{}|{}".format(dev, dtype, engine, ((n + 255) // 256) * 256)


def time_getrf(n, dtype="c64", engine=1, la_nb=0, reps=2, seed=0):
    """Milliseconds per factorisation of a seeded random n x n matrix with
    look-ahead width ``la_nb`` (CUDA events, after one warm-up)."""
    import torch
    code = nat.C64 if dtype == "c64" else nat.C128
    tdt = torch.complex64 if dtype == "c64" else torch.complex128
    gen = torch.Generator(device="cuda").manual_seed(seed)
    A0 = torch.randn(n, n, dtype=tdt, device="cuda", generator=gen) + 4 * torch.eye(n, dtype=tdt, device="cuda")
    A = torch.empty_like(A0)
    rowmap = torch.empty(n, dtype=torch.int32, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = int(nat.lib().bem200_getrf_workspace_size(code, engine, n))
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")

    def go():
        A.copy_(A0)
        nat.call("bem200_getrf_ex", code, engine, n, nat.ptr(A), n, nat.ptr(rowmap), nat.ptr(ipiv), nat.ptr(info),
                 nat.ptr(ws), wsb, 0, int(la_nb), nat.stream_ptr())
    go()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        go()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_lookahead(n, dtype="c64", engine=1, candidates=CANDIDATES, reps=2, use_cache=True):
    """The fastest look-ahead width for an n x n factorisation on this GPU
    (cached); returns (nb, {nb: ms})."""
    key = _key(dtype, engine, n)
    with _LOCK:
        if use_cache:
            if key in _MEM:
                return _MEM[key]["nb"], _MEM[key]["ms"]
            hit = _load().get(key)
            if hit:
                _MEM[key] = hit
                return hit["nb"], hit["ms"]
        cands = [c for c in candidates if 2 * c < n] or [min(candidates)]
        ms = {int(c): time_getrf(n, dtype, engine, c, reps) for c in cands}
        best = min(ms, key=ms.get)
        _MEM[key] = {"nb": best, "ms": {str(k): v for k, v in ms.items()}}
        _store(key, _MEM[key])
        return best, ms
