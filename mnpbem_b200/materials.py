"""Dielectric functions eps(lambda) and wavenumbers k = 2 pi / lambda * sqrt(eps).

Calling convention of the reference materials: ``eps, k = material(enei)``
with ``enei`` the vacuum wavelength in nm (reference
mnpbem/materials/eps_const.py:48-72, eps_drude.py:73-107, eps_table.py:114-152).
"""
import os

import numpy as np

#: eV <-> nm conversion used by the reference (mnpbem/utils/constants.py:9)
EV2NM = 1.0 / 8.0655477e-4


class EpsConst:
    """Wavelength-independent dielectric constant."""

    def __init__(self, eps):
        if eps is None or not np.isscalar(eps):
            raise TypeError("EpsConst: 'eps' must be a numeric value")
        self.eps = eps

    def __call__(self, enei):
        enei = np.asarray(enei)
        eps = np.full_like(enei, self.eps, dtype=complex)
        return eps, 2 * np.pi / enei * np.sqrt(eps)

    def __repr__(self):
        return "EpsConst({})".format(self.eps)


class EpsDrude:
    """Drude metal eps = eps0 - wp^2 / (w (w + i gammad)), energies in eV.

    ``EpsDrude.gold()``, ``.silver()``, ``.aluminum()`` give MNPBEM's preset
    metals: a free-electron (jellium) plasma energy from the electron-gas
    parameter rs, wp = sqrt(4 pi n) Hartree with n = 3 / (4 pi rs^3) in atomic
    units, and the toolbox's background eps0 and damping (reference
    mnpbem/materials/eps_drude.py:126-217, MATLAB @epsdrude/init.m)."""

    _HARTREE = 27.2116        # eV
    _PRESETS = {              # rs, eps0, damping in Hartree
        "gold": (3.0, 10.0, 0.66 / 27.2116 / 10), "silver": (3.0, 3.3, 0.66 / 27.2116 / 30),
        "aluminum": (2.07, 1.0, 1.06 / 27.2116)}
    _ALIASES = {"Au": "gold", "Ag": "silver", "Al": "aluminum"}

    def __init__(self, eps0, wp, gammad, name=None):
        self.eps0, self.wp, self.gammad, self.name = eps0, wp, gammad, name

    @classmethod
    def from_name(cls, name):
        key = cls._ALIASES.get(name, name)
        if key not in cls._PRESETS:
            raise ValueError("Material name unknown: {}".format(name))
        rs, eps0, gam = cls._PRESETS[key]
        wp = np.sqrt(4 * np.pi * (3 / (4 * np.pi * rs ** 3)))
        return cls(eps0=eps0, wp=wp * cls._HARTREE, gammad=gam * cls._HARTREE, name=name)

    @classmethod
    def gold(cls):
        return cls.from_name("gold")

    @classmethod
    def silver(cls):
        return cls.from_name("silver")

    @classmethod
    def aluminum(cls):
        return cls.from_name("aluminum")

    def __call__(self, enei):
        enei = np.asarray(enei, dtype=float)
        w = EV2NM / enei
        eps = self.eps0 - self.wp ** 2 / (w * (w + 1j * self.gammad))
        return eps, 2 * np.pi / enei * np.sqrt(eps)

    def __repr__(self):
        return "EpsDrude({}, {}, {})".format(self.eps0, self.wp, self.gammad)


def _bundled_tables():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "eps_tables.npz")
    return np.load(path) if os.path.exists(path) else {}


class EpsTable:
    """Tabulated refractive index (columns: energy [eV], n, k), cubic-spline
    interpolated in wavelength; eps = (n + i k)^2.  Raises ValueError outside
    the tabulated range, like the reference (mnpbem/materials/eps_table.py).

    ``filename`` is a path, or the name of one of the tables the reference
    ships: 'gold.dat', 'silver.dat' (Johnson & Christy), 'goldpalik.dat',
    'silverpalik.dat', 'copperpalik.dat' (Palik)."""

    def __init__(self, filename):
        from scipy.interpolate import CubicSpline
        if os.path.exists(filename):
            rows = []
            with open(filename) as f:
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
            data = np.array(rows)
        else:
            tables = _bundled_tables()
            name = os.path.basename(filename)
            if name not in tables:
                raise FileNotFoundError("Material data file not found: {}".format(filename))
            data = np.asarray(tables[name])
        if len(data) == 0:
            raise ValueError("No valid data found in {}".format(filename))
        self.filename = os.path.basename(filename)
        enei = EV2NM / data[:, 0]
        order = np.argsort(enei)
        self.enei = enei[order]
        self.ni = CubicSpline(self.enei, data[order, 1])
        self.ki = CubicSpline(self.enei, data[order, 2])

    def __call__(self, enei):
        enei = np.asarray(enei, dtype=float)
        if np.any(enei < self.enei.min()) or np.any(enei > self.enei.max()):
            raise ValueError("Wavelength out of range. Valid range: {:.1f} - {:.1f} nm".format(
                self.enei.min(), self.enei.max()))
        eps = (self.ni(enei) + 1j * self.ki(enei)) ** 2
        return eps, 2 * np.pi / enei * np.sqrt(eps)


class EpsValues:
    """Dielectric function given by a lookup {wavelength: eps}; used to drive a
    solve with eps values computed elsewhere (e.g. sampled from a table)."""

    def __init__(self, table):
        self.table = {float(k): complex(v) for k, v in dict(table).items()}

    def __call__(self, enei):
        e = float(np.asarray(enei).ravel()[0])
        for key, val in self.table.items():
            if abs(key - e) <= 1e-9 * max(1.0, abs(e)):
                eps = np.asarray(val, dtype=complex)
                return eps, 2 * np.pi / np.asarray(enei, dtype=float) * np.sqrt(eps)
        raise ValueError("EpsValues: no value tabulated at {} nm".format(e))
