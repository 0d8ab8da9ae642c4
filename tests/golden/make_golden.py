"""Generate the golden fixtures in this directory from the reference MNPBEM.

Runs the UNMODIFIED reference Python package (import-only stand-ins for its
absent plotting dependencies are installed by ``_refenv``) and stores small
input/output vectors that pin the oracle and the geometry module:

* ``geom_spheres.npz``  : face arrays of trisphere(144, 20) and a sample of
                          trisphere(1444, 40) incl. quadrature points.
* ``refined_cfg0.npz``  : refinement coefficients (after the closed-surface
                          correction) of trisphere(144, 20), every 4th entry.
* ``matrices_s60.npz``  : dense G1, G2, H1, H2 and the solution of
                          trisphere(32, 10) (60 faces) in water, Drude gold, 600 nm.
* ``spectrum_cfg0.npz`` : ext / sca of trisphere(144, 20), vacuum, Drude gold,
                          41 wavelengths 400-800 nm, x-pol along +z.
* ``dimer_small.npz``   : 2 x trisphere(144, 10), 2 nm gap on x, water, Drude
                          gold: ext/sca at 3 wavelengths, sig at 620 nm.
* ``matlab_cfg0.npz``   : MNPBEM17 MATLAB ext/sca/abs of trisphere(144, 20) with
                          tabulated gold (validation/03_bemret/sphere/data/
                          bemret_matlab.csv) and the reference EpsTable('gold.dat')
                          eps at those wavelengths.
* ``dimer_cfg1.npz``    : ext / sca of the 5768-face dimer (2 x trisphere(1444, 40),
                          +-21 nm on x, water, Drude gold) at 650 nm, plus
                          checksums of sig (slow: ~1 min).
* ``hmat_trees.npz``    : reference cluster trees, admissibility block lists and
                          ACA ranks / errors for the sphere and the small dimer.
* ``meshes.npz``        : face arrays of the reference mesh generators; ext / sca of a
                          small curved rod, rounded cube and flat ellipsoid.
* ``matlab_rod.npz``    : MNPBEM17 MATLAB and reference-Python ext / sca of the gold rod
                          trirod(10, 40, [15, 15, 15]) (validation/03_bemret/rod) and the
                          tabulated-gold eps at those wavelengths.
* ``matlab_iter.npz``   : MNPBEM17 MATLAB direct and iterative (bemiter) ext of
                          trisphere(144, 20) with tabulated gold (validation/08_iterative).
* ``eps_tables.npz``    : eps and k of the reference EpsTable for each of its five tables,
                          and the parameters of its preset Drude metals.
* ``planewave_field.npz`` : PlaneWaveRet.field of the reference on a small curved rod.
* ``editing.npz``       : Particle.rot and ComParticle shift / scale / rot / ipart of the reference.
* ``shape_fd_rod.npz``  : the reference solver's central-difference derivatives of the extinction
                          of a small curved rod along seeded vertex directions (h = 1e-4 nm).
* ``field_potential.npz`` : BEMRet.potential / .field inside and outside and slices of the
                          Cartesian-derivative Green functions (Gp, H1p, H2p) of the small dimer
                          (two polarisations) and the vacuum sphere.

Usage:  MNPBEM_REFERENCE=<reference checkout> python tests/golden/make_golden.py [--skip-cfg1] [--hmat-only]
        [--meshes-only] [--field-only] [--shape-only]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refenv  # noqa: E402

_refenv.setup()
from mnpbem.bem import BEMRet  # noqa: E402
from mnpbem.geometry import ComParticle, Particle, trisphere  # noqa: E402
from mnpbem.materials import EpsConst, EpsDrude, EpsTable  # noqa: E402
from mnpbem.simulation import PlaneWaveRet  # noqa: E402

DRUDE_AU = (9.84, 9.0, 0.067)
POL = np.array([[1.0, 0.0, 0.0]])
DIR = np.array([[0.0, 0.0, 1.0]])


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print("wrote", name, os.path.getsize(path), "bytes")


def geom():
    out = {}
    for tag, n, d, sample in (("s144", 144, 20.0, None), ("s1444", 1444, 40.0, np.arange(0, 2884, 97))):
        p = trisphere(n, d)
        ind = np.arange(p.nfaces) if sample is None else sample
        for a in ("pos", "nvec", "tvec1", "tvec2", "area"):
            out[tag + "_" + a] = getattr(p, a)[ind]
        out[tag + "_bradius"] = p.bradius()[ind]
        out[tag + "_ind"] = ind
        sub = ind[:12]
        qp, qw, qr = p.quadpol(sub)
        out[tag + "_quadpol_pos"], out[tag + "_quadpol_w"], out[tag + "_quadpol_row"] = qp, qw, qr
        qp, qw, qr = Particle.quad(p, sub)
        out[tag + "_quad_pos"], out[tag + "_quad_w"], out[tag + "_quad_row"] = qp, np.asarray(qw.sum(axis=0)).ravel(), qr
    save("geom_spheres.npz", **out)


def refined_cfg0():
    p = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20)], [[2, 1]], 1, interp="curv")
    bem = BEMRet(p)
    r = bem.g.g[0][0].refined
    sel = np.arange(0, len(r.row), 4)
    save("refined_cfg0.npz", row=r.row[sel], col=r.col[sel], g=r.g.real[sel], f=r.f.real[sel],
         nref=len(r.row), gsum=np.sum(np.abs(r.g)), fsum=np.sum(np.abs(r.f)))


def matrices_s60():
    p = ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [trisphere(32, 10)], [[2, 1]], 1, interp="curv")
    bem = BEMRet(p)
    enei = 600.0
    g = bem.g
    G1 = g.eval(0, 0, "G", enei)
    G2 = g.eval(1, 1, "G", enei)
    H1 = g.eval(0, 0, "H1", enei)
    H2 = g.eval(1, 1, "H2", enei)
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(p, enei))
    save("matrices_s60.npz", enei=enei, G1=G1, G2=G2, H1=H1, H2=H2, sig1=sig.sig1, sig2=sig.sig2,
         h1=sig.h1, h2=sig.h2, Sigma1=bem.Sigma1, ext=exc.extinction(sig), sca=exc.scattering(sig)[0])


def spectrum_cfg0():
    p = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20)], [[2, 1]], 1, interp="curv")
    bem = BEMRet(p)
    exc = PlaneWaveRet(POL, DIR)
    enei = np.linspace(400, 800, 41)
    ext = np.zeros(41)
    sca = np.zeros(41)
    t0 = time.time()
    for i, e in enumerate(enei):
        sig, bem = bem.solve(exc.potential(p, e))
        ext[i] = exc.extinction(sig)
        sca[i] = exc.scattering(sig)[0]
        if i == 20:
            s20 = sig
    save("spectrum_cfg0.npz", enei=enei, ext=ext, sca=sca, seconds=time.time() - t0,
         sig1_600=s20.sig1, sig2_600=s20.sig2, h1_600=s20.h1, h2_600=s20.h2)


def _dimer(n, dia, gap_half):
    a, b = trisphere(n, dia), trisphere(n, dia)
    a.shift([-(dia / 2 + gap_half), 0, 0])
    b.shift([dia / 2 + gap_half, 0, 0])
    return ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")


def dimer_small():
    p = _dimer(144, 10.0, 1.0)
    bem = BEMRet(p)
    exc = PlaneWaveRet(POL, DIR)
    enei = np.array([520.0, 620.0, 720.0])
    ext, sca = [], []
    for e in enei:
        sig, bem = bem.solve(exc.potential(p, e))
        ext.append(exc.extinction(sig))
        sca.append(exc.scattering(sig)[0])
        if e == 620.0:
            s = sig
    r01 = bem.g.g[0][1].refined
    save("dimer_small.npz", enei=enei, ext=np.array(ext), sca=np.array(sca), sig1=s.sig1, sig2=s.sig2,
         h1=s.h1, h2=s.h2, cross_row=r01.row, cross_col=r01.col, cross_g=r01.g.real, cross_f=r01.f.real)


def matlab_cfg0():
    csv = os.path.join(_refenv.REFERENCE_ROOT, "validation", "03_bemret", "sphere", "data", "bemret_matlab.csv")
    data = np.loadtxt(csv, delimiter=",", skiprows=1)
    gold = EpsTable("gold.dat")
    eps = np.array([complex(np.asarray(gold(e)[0]).ravel()[0]) for e in data[:, 0]])
    save("matlab_cfg0.npz", enei=data[:, 0], ext=data[:, 1], sca=data[:, 2], absorption=data[:, 3], eps_gold=eps)


def matlab_rod():
    """MNPBEM17 (MATLAB) and reference-Python ext / sca of the curved gold rod
    trirod(10, 40, [15, 15, 15]) in vacuum, tabulated gold, x-pol along +z and
    z-pol along +x, 41 wavelengths 400-800 nm
    (validation/03_bemret/rod/data/bemret_{matlab,python}.csv), with the
    reference EpsTable('gold.dat') eps at those wavelengths."""
    d = os.path.join(_refenv.REFERENCE_ROOT, "validation", "03_bemret", "rod", "data")
    m = np.loadtxt(os.path.join(d, "bemret_matlab.csv"), delimiter=",", skiprows=1)
    p = np.loadtxt(os.path.join(d, "bemret_python.csv"), delimiter=",", skiprows=1)
    gold = EpsTable("gold.dat")
    eps = np.array([complex(np.asarray(gold(e)[0]).ravel()[0]) for e in m[:, 0]])
    save("matlab_rod.npz", enei=m[:, 0], matlab=m[:, 1:], python=p[:, 1:], eps_gold=eps,
         columns=np.array(["ext_x", "sca_x", "ext_z", "sca_z"]))


def matlab_iter():
    """MNPBEM17 (MATLAB) direct and iterative (bemiter) retarded extinction of
    trisphere(144, 20) in vacuum with tabulated gold, x-pol along +z, 41
    wavelengths 400-800 nm (validation/08_iterative/sphere/data/ret_matlab.csv)."""
    csv = os.path.join(_refenv.REFERENCE_ROOT, "validation", "08_iterative", "sphere", "data", "ret_matlab.csv")
    m = np.loadtxt(csv, delimiter=",", skiprows=1)
    gold = EpsTable("gold.dat")
    eps = np.array([complex(np.asarray(gold(e)[0]).ravel()[0]) for e in m[:, 0]])
    save("matlab_iter.npz", enei=m[:, 0], ext_direct=m[:, 1], ext_iter=m[:, 2], eps_gold=eps)


def eps_tables():
    """eps and k of the reference EpsTable for every table it ships, at 25
    wavelengths inside each table's range."""
    out = {}
    for name in ("gold.dat", "silver.dat", "goldpalik.dat", "silverpalik.dat", "copperpalik.dat"):
        t = EpsTable(name)
        lo, hi = float(t.enei.min()), float(t.enei.max())
        enei = np.linspace(lo + 1e-6 * (hi - lo), hi - 1e-6 * (hi - lo), 25)
        eps, k = t(enei)
        key = name.replace(".dat", "")
        out[key + "_enei"], out[key + "_eps"], out[key + "_k"] = enei, np.asarray(eps), np.asarray(k)
    for metal in ("gold", "silver", "aluminum"):
        m = getattr(EpsDrude, metal)()
        out["drude_" + metal] = np.array([m.eps0, m.wp, m.gammad])
    save("eps_tables.npz", **out)


def planewave_field():
    """PlaneWaveRet.field of the reference (x-pol along +z, z-pol along +x) on
    the small curved rod trirod(12, 30, [9, 5, 5]) in water, inside and outside."""
    from mnpbem.geometry import mesh_generators as mg
    part = mg.trirod(12.0, 30.0, [9, 5, 5], interp="curv")
    p = ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [part], [[2, 1]], 1, interp="curv")
    exc = PlaneWaveRet(np.array([[1.0, 0, 0], [0, 0, 1.0]]), np.array([[0, 0, 1.0], [1.0, 0, 0]]))
    out = {}
    for inout in (1, 2):
        f = exc.field(p, 600.0, inout=inout)
        out["e%d" % inout], out["h%d" % inout] = f.e, f.h
    save("planewave_field.npz", **out)


def editing():
    """Particle.rot and the ComParticle editing methods of the reference on
    two curved spheres: rot(30 deg, [1, 1, 0]) of one, then the compound
    shifted, scaled and rotated; ipart of a few global faces."""
    a, b = trisphere(60, 10.0), trisphere(32, 6.0)
    a.rot(30.0, [1.0, 1.0, 0.0])
    b.shift([9.0, 0.0, 0.0])
    p = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")
    out = {"rot_pos": a.pos, "rot_nvec": a.nvec, "rot_area": a.area}
    p.shift([1.0, -2.0, 0.5])
    p.scale(1.5)
    p.rot(45.0, [0.0, 0.0, 1.0])
    out.update(cp_pos=p.pos, cp_nvec=p.nvec, cp_area=p.area)
    ind = np.array([0, 5, 115, 116, 150, 175])
    pi, li = p.ipart(ind)
    out.update(ipart_ind=ind, ipart_part=np.asarray(pi), ipart_local=np.asarray(li))
    save("editing.npz", **out)


def dimer_cfg1():
    p = _dimer(1444, 40.0, 1.0)
    t0 = time.time()
    bem = BEMRet(p)
    t1 = time.time()
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(p, 650.0))
    t2 = time.time()
    ext = exc.extinction(sig)
    sca = exc.scattering(sig)[0]
    nref = [len(bem.g.g[i][j].refined.row) for i in range(2) for j in range(2)]
    save("dimer_cfg1.npz", enei=650.0, ext=ext, sca=sca, nref=np.array(nref),
         sig1_abs_sum=np.sum(np.abs(sig.sig1)), sig2_abs_sum=np.sum(np.abs(sig.sig2)),
         h1_abs_sum=np.sum(np.abs(sig.h1)), h2_abs_sum=np.sum(np.abs(sig.h2)),
         sig2_head=sig.sig2[:64], ctor_s=t1 - t0, solve_s=t2 - t1)


def field_potential():
    """BEMRet.potential / BEMRet.field (reference bem_ret.py:1833-1895 via
    CompGreenRet.potential / .field, compgreen_ret.py:912-1038) inside and
    outside, for the reference's own solutions: the small dimer at 620 nm with
    two polarisations and the vacuum sphere at 600 nm; plus slices and sums of
    the Cartesian-derivative Green functions (eval keys Gp, H1p, H2p)."""
    out = {}
    cases = (("dimer", _dimer(144, 10.0, 1.0), 620.0, np.array([[1.0, 0, 0], [0, 1.0, 0]]),
              np.array([[0, 0, 1.0], [0, 0, 1.0]])),
             ("sphere", ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20)], [[2, 1]], 1,
                                    interp="curv"), 600.0, POL, DIR))
    for tag, p, enei, pol, dirs in cases:
        bem = BEMRet(p)
        exc = PlaneWaveRet(pol, dirs)
        sig, bem = bem.solve(exc.potential(p, enei))
        out[tag + "_enei"] = enei
        for k in ("sig1", "sig2", "h1", "h2"):
            out[tag + "_" + k] = getattr(sig, k)
        for io in (1, 2):
            pot = bem.potential(sig, io)
            for k in ("phi", "phip", "a", "ap"):
                name = k[:-1] + str(io) + "p" if k.endswith("p") and k != "phi" else k + str(io)
                if k == "phip":
                    name = "phi{}p".format(io)
                out["{}_pot{}_{}".format(tag, io, k)] = getattr(pot, name)
            f = bem.field(sig, io)
            out["{}_field{}_e".format(tag, io)] = f.e
            out["{}_field{}_h".format(tag, io)] = f.h
        for (i, j, key) in ((0, 0, "H1p"), (1, 1, "H2p"), (1, 1, "Gp"), (0, 0, "Gp")):
            M = bem.g.eval(i, j, key, enei)
            nm = "{}_{}{}{}".format(tag, key, i, j)
            out[nm + "_rows"] = np.asarray(M)[:8]
            out[nm + "_abssum"] = np.sum(np.abs(M))
    save("field_potential.npz", **out)


def shape_fd():
    """The reference solver's own finite-difference derivatives of the
    extinction with respect to the vertices: trirod(12, 30, [9, 5, 5]) curved
    (96 faces, triangles and quads), gold in eps 1.77, 640 nm, x-polarised;
    central differences with step h = 1e-4 nm of the unmodified BEMRet along
    4 seeded unit directions in the space of the particle's verts2 (the nodes
    that fix the curved geometry; corner vertices stay, as in
    mnpbem_b200.shape.perturbed)."""
    from mnpbem.geometry import trirod

    def build(delta):
        part = trirod(12.0, 30.0, [9, 5, 5], interp="curv")
        if delta is not None:
            part.verts2 = part.verts2 + delta
            part._norm()
        return ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [part], [[2, 1]], 1, interp="curv")

    p0 = build(None)
    v2 = p0.p[0].verts2.copy()
    rng = np.random.default_rng(11)
    D = rng.standard_normal((4,) + v2.shape)
    D /= np.sqrt(np.sum(D * D, axis=(1, 2), keepdims=True))
    h, enei = 1e-4, 640.0
    exc = PlaneWaveRet(POL, DIR)

    def ext_of(p):
        bem = BEMRet(p)
        sig, _ = bem.solve(exc.potential(p, enei))
        return exc.extinction(sig)

    ext0 = ext_of(p0)
    dext = np.array([(ext_of(build(h * d)) - ext_of(build(-h * d))) / (2 * h) for d in D])
    save("shape_fd_rod.npz", verts2=v2, D=D, h=h, enei=enei, ext=ext0, dext=dext)


def hmat_trees():
    """Cluster trees, block partitions and ACA ranks of the reference H-matrix
    (mnpbem/greenfun/clustertree.py, hmatrix.py) for the sphere (cleaf 32,
    eta 1) and the small dimer (cleaf 64, eta 2.5), with the wavenumber-aware
    admissibility at 600 nm and ACA (htol 1e-6, kmax 100) of the dense G1 = G11 - G21
    (vacuum sphere: G11 alone) at 600 nm."""
    from mnpbem.greenfun.clustertree import ClusterTree
    from mnpbem.greenfun.hmatrix import HMatrix, make_kaware_fadmiss
    out = {}
    enei = 600.0
    cases = (("s", ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20)], [[2, 1]], 1,
                               interp="curv"), 32, 1.0),
             ("d", _dimer(144, 10.0, 1.0), 64, 2.5))
    for tag, p, cleaf, eta in cases:
        ip = None
        if len(p.p) > 1:
            ip = np.concatenate([np.full(q.n, i) for i, q in enumerate(p.p)])
        tree = ClusterTree(p.pos, cleaf=cleaf, ipart_arr=ip)
        out[tag + "_son"], out[tag + "_cind"], out[tag + "_ind"] = tree.son, tree.cind, tree.ind
        out[tag + "_mid"], out[tag + "_rad"], out[tag + "_ipart"] = tree.mid, tree.rad, tree.ipart
        h = HMatrix(tree=tree, htol=1e-6, kmax=100, fadmiss=make_kaware_fadmiss(2 * np.pi / enei, eta0=eta))
        out[tag + "_row1"], out[tag + "_col1"] = h.row1, h.col1
        out[tag + "_row2"], out[tag + "_col2"] = h.row2, h.col2
        bem = BEMRet(p)
        G = bem.g.eval(0, 0, "G", enei)
        G21 = bem.g.eval(1, 0, "G", enei)
        if not np.isscalar(G21):
            G = G - G21
        h.aca(lambda r, c: G[r, c])
        out[tag + "_ranks"] = np.array([u.shape[1] for u in h.lhs])
        full = h.full(xp=np) if "xp" in h.full.__code__.co_varnames else h.full()
        out[tag + "_aca_err"] = np.linalg.norm(full - G) / np.linalg.norm(G)
    save("hmat_trees.npz", **out)


MESH_CASES = (
    # tag, generator, args, kwargs, store every face (else a sample)
    ("ell", "triellipsoid", (400, [10.0, 15.0, 25.0]), {}, True),
    ("seg", "trispheresegment", (np.linspace(0, np.pi, 7), np.linspace(0, np.pi / 2, 5), 10.0),
     {"triangles": True, "interp": "curv"}, True),
    ("rod", "trirod", (20.0, 60.0, [13, 6, 9]), {"interp": "curv"}, True),
    ("rodtri", "trirod", (12.0, 30.0, [9, 5, 5]), {"triangles": True, "interp": "curv"}, True),
    ("cube", "tricube", (6, 40.0, 0.25), {"interp": "curv"}, True),
    ("rod2400", "trirod", (20.0, 80.0, [41, 16, 31]), {"interp": "curv"}, False),
    ("cube25k", "tricube", (66, 100.0, 0.25), {"interp": "curv"}, False),
)


def _face_nodes(p):
    """Per-face node coordinates (n, 9, 3), NaN where a face has no such node."""
    if p.faces2 is None:
        f, v = p.faces, p.verts
    else:
        f, v = p.faces2, p.verts2
    out = np.full((len(f), 9, 3), np.nan)
    ok = ~np.isnan(f)
    out[:, :f.shape[1]][ok] = v[f[ok].astype(int)]
    return out


def meshes():
    """Face arrays of the reference mesh generators (triellipsoid, trispheresegment,
    trirod, tricube), and ext / sca of a small curved rod, a rounded cube and a
    flat ellipsoid (water, Drude gold; x-pol along +z and z-pol along +x) from
    the reference BEMRet."""
    from mnpbem.geometry import mesh_generators as mg
    out = {}
    for tag, name, args, kw, full in MESH_CASES:
        p = getattr(mg, name)(*args, **kw)
        ind = np.arange(p.nfaces) if full else np.arange(0, p.nfaces, max(1, p.nfaces // 40))
        out[tag + "_nfaces"] = p.nfaces
        out[tag + "_nverts"] = p.nverts
        out[tag + "_ntri"] = int(np.sum(np.isnan(p.faces[:, 3])))
        out[tag + "_ind"] = ind
        for a in ("pos", "nvec", "tvec1", "area"):
            out[tag + "_" + a] = getattr(p, a)[ind]
        out[tag + "_bradius"] = p.bradius()[ind]
        out[tag + "_nodes"] = _face_nodes(p)[ind]
        out[tag + "_area_sum"] = np.sum(p.area)
        out[tag + "_pos_sum"] = np.sum(p.pos, axis=0)
    for tag, name, args, interp in (("rodbem", "trirod", (12.0, 30.0, [9, 5, 5]), "curv"),
                                    ("cubebem", "tricube", (5, 20.0, 0.25), "curv"),
                                    ("ellbem", "triellipsoid", (60, [4.0, 6.0, 9.0]), "flat")):
        part = getattr(mg, name)(*args) if interp == "flat" else getattr(mg, name)(*args, interp=interp)
        p = ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [part], [[2, 1]], 1, interp=interp)
        bem = BEMRet(p)
        exc = PlaneWaveRet(np.array([[1.0, 0, 0], [0, 0, 1.0]]), np.array([[0, 0, 1.0], [1.0, 0, 0]]))
        enei = np.array([560.0, 640.0])
        ext, sca = [], []
        for e in enei:
            sig, bem = bem.solve(exc.potential(p, e))
            ext.append(exc.extinction(sig))
            sca.append(exc.scattering(sig)[0])
        out[tag + "_enei"], out[tag + "_ext"], out[tag + "_sca"] = enei, np.array(ext), np.array(sca)
        out[tag + "_nfaces"] = p.nfaces
        out[tag + "_sig2"] = sig.sig2
    save("meshes.npz", **out)


if __name__ == "__main__":
    if "--field-only" in sys.argv:
        field_potential()
        sys.exit(0)
    if "--shape-only" in sys.argv:
        shape_fd()
        sys.exit(0)
    if "--meshes-only" in sys.argv:
        meshes()
        matlab_rod()
        matlab_iter()
        eps_tables()
        planewave_field()
        editing()
        sys.exit(0)
    hmat_trees()
    if "--hmat-only" in sys.argv:
        sys.exit(0)
    meshes()
    matlab_rod()
    matlab_iter()
    eps_tables()
    planewave_field()
    editing()
    geom()
    refined_cfg0()
    matrices_s60()
    spectrum_cfg0()
    dimer_small()
    matlab_cfg0()
    field_potential()
    shape_fd()
    if "--skip-cfg1" not in sys.argv:
        dimer_cfg1()
