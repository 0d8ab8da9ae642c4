"""Wavelength sweep on the GPU against the reference's 41-wavelength spectrum
(tests/golden/spectrum_cfg0.npz: trisphere(144, 20) in vacuum, Drude gold)."""
import numpy as np
import pytest

from conftest import golden
from meshes import sphere

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_spectrum_matches_reference(cuda, precision):
    from mnpbem_b200.spectrum import solve_spectrum
    g = golden("spectrum_cfg0.npz")
    res = solve_spectrum(sphere(), g["enei"], [[1.0, 0, 0]], [[0, 0, 1.0]], precision=precision)
    assert res["ext"].shape == (41, 1)
    assert np.max(np.abs(res["ext"][:, 0] - g["ext"]) / g["ext"]) < 1e-10
    assert np.max(np.abs(res["sca"][:, 0] - g["sca"]) / g["sca"]) < 1e-10
