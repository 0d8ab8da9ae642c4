"""Failure reporting of the mixed-precision solve (no GPU fault involved:
every case is an ordinary argument or input that the library must turn into
an error status).

* refinement that cannot reach its tolerance returns BEM200_ERR_NOCONV and
  BEMRet raises RuntimeError instead of returning the unconverged iterate;
* with gmres_ir=True the same stalled refinement continues as GMRES-IR and
  reaches the FP64 solution;
* factors with an exactly zero pivot give BEM200_ERR_SINGULAR.
"""
import ctypes

import numpy as np
import pytest

from meshes import dimer, sphere

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def test_unconverged_refinement_raises(cuda):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = sphere()
    exc = PlaneWaveRet(POL, DIR)
    bem = BEMRet(cp, precision="mixed", ir_maxit=1, ir_tol=1e-30, gmres_ir=False)
    with pytest.raises(RuntimeError, match="status 6"):
        bem.solve(exc.potential(cp, 600.0))
    with pytest.raises(RuntimeError, match="status 6"):
        bem.cross_sections(exc, 600.0)


def test_gmres_ir_continues_stalled_refinement(cuda):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = dimer()
    exc = PlaneWaveRet(POL, DIR)
    sig64, _ = BEMRet(cp).solve(exc.potential(cp, 620.0))
    ext64 = exc.extinction(sig64)
    bem = BEMRet(cp, precision="mixed", ir_maxit=1, ir_tol=1e-12, gmres_ir=True)
    sig, bem = bem.solve(exc.potential(cp, 620.0))
    assert bem.last_ir[2] == "gmres-ir" and bem.last_ir[1] <= 1e-12, bem.last_ir
    assert abs(exc.extinction(sig) - ext64) / abs(ext64) < 1e-10
    # an unreachable tolerance after GMRES-IR still raises
    bem2 = BEMRet(cp, precision="mixed", ir_maxit=1, ir_tol=1e-30, gmres_ir=True, gmres_maxit=3)
    with pytest.raises(RuntimeError, match="did not converge"):
        bem2.solve(exc.potential(cp, 620.0))


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_zero_pivot_reports_singular(cuda, precision):
    """G1 with a zero column: the init's zero-pivot check returns
    BEM200_ERR_SINGULAR (3) for both precisions."""
    import torch
    from mnpbem_b200 import _native as nat
    L = nat.lib()
    n = 96
    dt = torch.complex128 if precision == 0 else torch.complex64
    ws = torch.zeros(int(L.bem200_bem_workspace_size(precision, n)), dtype=torch.uint8, device=cuda)
    slots = [ctypes.c_void_p() for _ in range(4)]
    nat.call("bem200_bem_slots", precision, n, nat.ptr(ws), *[ctypes.byref(s) for s in slots])
    esz = 16 if precision == 0 else 8

    def slot(addr):  # the n x n matrix at a workspace slot, as a view of ws
        off = addr - ws.data_ptr()
        return ws[off:off + n * n * esz].view(dt).view(n, n)

    g = torch.Generator(device="cpu").manual_seed(5)
    for s_ in slots:
        m = torch.randn(n, n, generator=g, dtype=torch.complex128) / n + 4 * torch.eye(n)
        slot(s_.value).copy_(m.to(dt))
    slot(slots[0].value)[:, 7] = 0  # column 7 of G1
    nvec = torch.zeros((n, 3), dtype=torch.float64, device=cuda)
    nvec[:, 2] = 1
    e1 = (ctypes.c_double * 2)(1.0, 0.0)
    e2 = (ctypes.c_double * 2)(-10.0, 1.0)
    engine = 1 if precision else 0
    gb = int(L.bem200_gemm_workspace_size(engine, n, n, n)) + 256
    gws = torch.empty(gb, dtype=torch.uint8, device=cuda)
    info = ctypes.c_int32(0)
    st = L.bem200_bem_init(precision, engine, n, nat.ptr(ws), 0, e1, e2, nat.ptr(nvec), 0.01, nat.ptr(gws), gb,
                           ctypes.byref(info), nat.stream_ptr())
    assert st == nat.ERR_SINGULAR and info.value == 8, (st, info.value, nat.last_error())
