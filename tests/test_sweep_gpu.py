"""The uneven-mesh sweep on the GPU: worker threads run on the caller's device
and their results equal single solves of the same (mesh, wavelength) units."""
import numpy as np
import pytest

from meshes import dimer, sphere

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0], [0, 1.0, 0]])
DIR = np.array([[0, 0, 1.0], [0, 0, 1.0]])


@pytest.mark.parametrize("schedule", ["interleave", "mesh"])
def test_solve_sweep_two_workers(cuda, schedule):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.sweep import solve_sweep
    parts = [sphere(), dimer()]
    enei = np.array([560.0, 610.0, 660.0])
    r = solve_sweep(parts, enei, POL, DIR, precision="mixed", workers=2, schedule=schedule)
    exc = PlaneWaveRet(POL, DIR)
    for m, cp in enumerate(parts):
        bem = BEMRet(cp, precision="fp64")
        for i, lam in enumerate(enei):
            ref = bem.cross_sections(exc, float(lam))
            assert np.max(np.abs(r["ext"][m, i] - ref["ext"]) / np.abs(ref["ext"])) < 1e-10
            assert np.max(np.abs(r["sca"][m, i] - ref["sca"]) / np.abs(ref["sca"])) < 1e-10
    assert r["solves"] == len(parts) * len(enei) * len(POL)
