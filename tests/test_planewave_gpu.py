"""Plane-wave right-hand side and far fields on the GPU against the host
path (which follows the reference, pinned by the golden spectra)."""
import numpy as np
import pytest

from conftest import golden
from meshes import dimer, rel, sphere

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mk", [sphere, dimer], ids=["sphere", "dimer"])
def test_rhs_device_matches_host(cuda, mk):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = mk()
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    exc = PlaneWaveRet(pol, dirs)
    bem = BEMRet(cp)
    enei = 610.0
    bem._eps(enei)
    b_host, npol = bem.rhs(exc.potential(cp, enei))
    b_dev, npol2 = exc.rhs_device(cp, enei, bem._eps_mode, bem._e1p, bem._e2p)
    assert npol == npol2 == 2
    assert rel(b_dev.cpu().numpy(), b_host) < 1e-14


def test_cross_sections_device_spectrum(cuda):
    """Fully on-device cross sections of the reference's 41-wavelength sphere spectrum."""
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    g = golden("spectrum_cfg0.npz")
    cp = sphere()
    exc = PlaneWaveRet([[1.0, 0, 0]], [[0, 0, 1.0]])
    bem = BEMRet(cp, precision="mixed")
    for i in range(0, 41, 8):
        out = bem.cross_sections(exc, float(g["enei"][i]))
        assert abs(out["ext"][0] - g["ext"][i]) / g["ext"][i] < 1e-10
        assert abs(out["sca"][0] - g["sca"][i]) / g["sca"][i] < 1e-10


def test_farfield_device_two_polarisations(cuda):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = dimer()
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    exc = PlaneWaveRet(pol, dirs)
    bem = BEMRet(cp)
    sig, _ = bem.solve(exc.potential(cp, 560.0))
    out = bem.cross_sections(exc, 560.0)
    assert rel(out["ext"], exc.extinction(sig)) < 1e-12
    assert rel(out["sca"], exc.scattering(sig)[0]) < 1e-12
