"""Oracle: the whole per-wavelength path, refinement to cross sections.

Test infrastructure only (see ``oracle/__init__.py``).
Mirrors the user-level sequence of the reference README (README.md:73-91):
BEMRet(p) -> bem.solve(exc.potential(p, enei)) -> exc.extinction / scattering.
"""
import os

import numpy as np

from . import bem as obem
from . import farfield as off
from . import green as ogreen


def pinfty():
    here = os.path.dirname(os.path.abspath(__file__))
    d = np.load(os.path.join(here, "..", "mnpbem_b200", "data", "pinfty256.npz"))
    return d["nvec"], d["area"]


class OracleBEM:
    """Refinement once per mesh, then per-wavelength Green matrices, init and solve."""

    def __init__(self, cp, order=5):
        self.cp = cp
        self.blocks = ogreen.refine_all(cp, order)

    def matrices(self, enei):
        return ogreen.bem_matrices(self.cp, self.blocks, enei)

    def solve(self, enei, pol, dirs, medium=1, return_state=False):
        cp = self.cp
        G1, G2, H1, H2 = self.matrices(enei)
        con = ogreen.connect(cp.inout)
        st = obem.bem_init(G1, G2, H1, H2, cp.eps1(enei), cp.eps2(enei), cp.nvec, enei,
                           con01_zero=bool(np.all(con[0][1] == 0)))
        exc = off.planewave_potential(cp, pol, dirs, enei, medium)
        phi, a, alpha, De = obem.excitation(st, exc, cp.eps1(enei), cp.eps2(enei))
        sig1, sig2, h1, h2 = obem.bem_solve(st, phi, a, alpha, De)
        ext = off.extinction(cp, sig1, sig2, h1, h2, enei, pol, dirs, medium)
        nv, ar = pinfty()
        sca = off.scattering(cp, sig1, sig2, h1, h2, enei, nv, ar, medium)
        out = dict(sig1=sig1, sig2=sig2, h1=h1, h2=h2, ext=ext, sca=sca)
        if return_state:
            out.update(G1=G1, G2=G2, H1=H1, H2=H2, state=st)
        return out
