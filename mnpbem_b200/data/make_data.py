"""Regenerate the mesh data files shipped in this directory.

``spheres.npz``   : vertex sets (unit-diameter-2 sphere, i.e. |v| = 1) and their
                    triangulations for the 24 vertex counts that ``trisphere``
                    accepts.  They are energy-minimised point distributions on
                    the sphere (R. Womersley); MNPBEM ships them as
                    ``mnpbem/data/sphere{n}_tri.bin`` (int32 nv, nf; float64 x, y,
                    z; int32 1-based faces).
``pinfty256.npz`` : the 256-direction unit sphere used for far-field
                    integration (directions, solid-angle weights, centroids),
                    shipped by MNPBEM as ``mnpbem/data/pinfty256.bin``.
``eps_tables.npz``: the tabulated optical constants (photon energy in eV, n, k)
                    that MNPBEM ships as ``mnpbem/materials/data/*.dat``: gold
                    and silver of Johnson & Christy, gold, silver and copper of
                    Palik.  ``EpsTable('gold.dat')`` reads them by name.

Run once in a checkout that has the MNPBEM sources next to it:
    python mnpbem_b200/data/make_data.py /path/to/MNPBEM
"""
import os
import sys

import numpy as np

NSAV = [32, 60, 144, 169, 225, 256, 289, 324, 361, 400, 441, 484,
        529, 576, 625, 676, 729, 784, 841, 900, 961, 1024, 1225, 1444]


def main(root):
    ddir = os.path.join(root, "mnpbem", "data")
    out = {}
    for n in NSAV:
        with open(os.path.join(ddir, "sphere{}_tri.bin".format(n)), "rb") as f:
            nv, nf = np.fromfile(f, dtype=np.int32, count=2)
            xyz = np.fromfile(f, dtype=np.float64, count=3 * nv).reshape(3, nv).T
            faces = np.fromfile(f, dtype=np.int32, count=3 * nf).reshape(nf, 3) - 1
        out["verts{}".format(n)] = xyz
        out["faces{}".format(n)] = faces.astype(np.int32)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "spheres.npz"), **out)
    with open(os.path.join(ddir, "pinfty256.bin"), "rb") as f:
        n = int(np.fromfile(f, dtype=np.int32, count=1)[0])
        rest = np.fromfile(f, dtype=np.float64)
    nvec = rest[:3 * n].reshape(3, n).T
    tail = rest[3 * n:]
    if tail.size == 4 * n:
        pos = tail[:3 * n].reshape(3, n).T
        area = tail[3 * n:]
    else:
        pos = nvec.copy()
        area = tail[:n]
    np.savez_compressed(os.path.join(here, "pinfty256.npz"), nvec=nvec, area=area, pos=pos)
    tables = {}
    mdir = os.path.join(root, "mnpbem", "materials", "data")
    for name in sorted(os.listdir(mdir)):
        if not name.endswith(".dat"):
            continue
        rows = []
        with open(os.path.join(mdir, name)) as f:
            for line in f:
                line = line.strip()
                if not line or line[0] in "%#":
                    continue
                try:
                    vals = [float(x) for x in line.split()]
                except ValueError:
                    continue
                if len(vals) >= 3:
                    rows.append(vals[:3])
        tables[name] = np.array(rows)
    np.savez_compressed(os.path.join(here, "eps_tables.npz"), **tables)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MNPBEM_REFERENCE")
    if not ref:
        sys.exit("usage: python make_data.py <path of the reference checkout> (or set MNPBEM_REFERENCE)")
    main(ref)
