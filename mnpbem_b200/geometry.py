"""Discretised particle surfaces (host side).

This module produces the per-face arrays that the GPU kernels consume:
centroids ``pos``, the orthonormal frame ``tvec1, tvec2, nvec``, areas,
bounding radii and the curved-element node coordinates from which the
quadrature points are generated on the device.  It mirrors the public surface
of the reference classes that sit in front of the retarded BEM path
(``Particle``, ``ComParticle``, ``trisphere``; reference
mnpbem/geometry/particle.py:249, mnpbem/geometry/comparticle.py:11,
mnpbem/geometry/mesh_generators.py:13) so that scripts written for the
reference build the same meshes here.

Faces are stored as in the reference: ``faces`` is (n, 4) float with NaN in
column 3 for triangles; curved particles additionally carry ``verts2`` and a
(n, 9) ``faces2`` table [v0 v1 v2 v3 e01 e12 e23|e20 e30 centre].
"""
import copy
import os

import numpy as np

from .quadrature import QuadFace

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

# ---------------------------------------------------------------------------
# shape functions (reference: mnpbem/geometry/particle.py:1606-1743)
# ---------------------------------------------------------------------------


def tri6_shape(x, y):
    """Quadratic 6-node triangle: corners (1,0), (0,1), (0,0) then edge midpoints."""
    l1, l2, l3 = x, y, 1 - x - y
    return np.stack([l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1),
                     4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1], axis=1)


def tri6_deriv(x, y):
    l1, l2, l3 = x, y, 1 - x - y
    z = np.zeros_like(x)
    dx = np.stack([4 * l1 - 1, z, -4 * l3 + 1, 4 * l2, -4 * l2, 4 * (l3 - l1)], axis=1)
    dy = np.stack([z, 4 * l2 - 1, -4 * l3 + 1, 4 * l1, 4 * (l3 - l2), -4 * l1], axis=1)
    return dx, dy


def quad4_shape(x, y):
    return np.stack([0.25 * (1 - x) * (1 - y), 0.25 * (1 + x) * (1 - y),
                     0.25 * (1 + x) * (1 + y), 0.25 * (1 - x) * (1 + y)], axis=1)


def quad4_deriv(x, y):
    dx = np.stack([-0.25 * (1 - y), 0.25 * (1 - y), 0.25 * (1 + y), -0.25 * (1 + y)], axis=1)
    dy = np.stack([-0.25 * (1 - x), -0.25 * (1 + x), 0.25 * (1 + x), 0.25 * (1 - x)], axis=1)
    return dx, dy


def quad9_shape(x, y):
    return np.stack([
        0.25 * x * (x - 1) * y * (y - 1), 0.25 * x * (x + 1) * y * (y - 1),
        0.25 * x * (x + 1) * y * (y + 1), 0.25 * x * (x - 1) * y * (y + 1),
        0.5 * (1 - x ** 2) * y * (y - 1), 0.5 * x * (x + 1) * (1 - y ** 2),
        0.5 * (1 - x ** 2) * y * (y + 1), 0.5 * x * (x - 1) * (1 - y ** 2),
        (1 - x ** 2) * (1 - y ** 2)], axis=1)


def quad9_deriv(x, y):
    dx = np.stack([
        0.25 * (2 * x - 1) * y * (y - 1), 0.25 * (2 * x + 1) * y * (y - 1),
        0.25 * (2 * x + 1) * y * (y + 1), 0.25 * (2 * x - 1) * y * (y + 1),
        -x * y * (y - 1), 0.5 * (2 * x + 1) * (1 - y ** 2),
        -x * y * (y + 1), 0.5 * (2 * x - 1) * (1 - y ** 2),
        -2 * x * (1 - y ** 2)], axis=1)
    dy = np.stack([
        0.25 * x * (x - 1) * (2 * y - 1), 0.25 * x * (x + 1) * (2 * y - 1),
        0.25 * x * (x + 1) * (2 * y + 1), 0.25 * x * (x - 1) * (2 * y + 1),
        0.5 * (1 - x ** 2) * (2 * y - 1), -x * (x + 1) * y,
        0.5 * (1 - x ** 2) * (2 * y + 1), -x * (x - 1) * y,
        -2 * (1 - x ** 2) * y], axis=1)
    return dx, dy


class Particle:
    """Faces and vertices of a discretised particle surface.

    ``Particle(verts, faces, interp='flat'|'curv')`` with ``faces`` of shape
    (n, 3) (triangles), (n, 4) (NaN in column 3 for triangles) or, together
    with ``verts2``, the 9-column curved face table (reference
    mnpbem/geometry/particle.py:310-399).
    """

    def __init__(self, verts, faces=None, interp="flat", norm=True, **kwargs):
        verts = np.asarray(verts, dtype=float).reshape(-1, 3)
        self.verts2 = None
        self.faces2 = None
        if faces is None:
            self.verts = verts
            self.faces = np.zeros((0, 4))
        else:
            faces = np.asarray(faces, dtype=float)
            if faces.ndim != 2:
                raise ValueError("Particle: 'faces' must be 2D; got {}D.".format(faces.ndim))
            if faces.shape[1] == 3:
                self.verts = verts
                self.faces = np.hstack([faces, np.full((faces.shape[0], 1), np.nan)])
            elif faces.shape[1] == 4:
                self.verts = verts
                self.faces = faces
            else:
                # curved table: extract the corner vertices
                self.verts2 = verts
                self.faces2 = faces
                corner = faces[:, :4].reshape(-1)
                valid = ~np.isnan(corner)
                uniq, inv = np.unique(corner[valid].astype(int), return_inverse=True)
                self.verts = verts[uniq]
                nf = np.full_like(faces[:, :4], np.nan)
                nf.flat[np.flatnonzero(valid)] = inv
                self.faces = nf
        self.quad = QuadFace(rule=kwargs.get("rule", 18), npol=kwargs.get("npol", (7, 5)),
                             refine=kwargs.get("refine", None))
        self.interp = interp
        if norm not in (False, "off") and len(self.faces) > 0:
            self._norm()
        else:
            self.pos = np.zeros((0, 3))
            self.vec = [np.zeros((0, 3))] * 3
            self.area = np.zeros(0)

    # ---------------------------------------------------------------- props
    @property
    def nvec(self):
        return self.vec[2]

    @property
    def tvec1(self):
        return self.vec[0]

    @property
    def tvec2(self):
        return self.vec[1]

    @property
    def nfaces(self):
        return self.faces.shape[0]

    n = nfaces

    @property
    def nverts(self):
        return self.verts.shape[0]

    def index34(self, ind=None):
        f = self.faces if ind is None else self.faces[np.asarray(ind)]
        tri = np.isnan(f[:, 3])
        return np.flatnonzero(tri), np.flatnonzero(~tri)

    # ---------------------------------------------------------------- norm
    def _norm(self):
        if self.interp == "flat":
            self._norm_flat()
        else:
            self._norm_curv()

    def _norm_flat(self):
        """Centroids, areas and frames of flat elements (reference particle.py:464-549)."""
        n = self.nfaces
        ind3, ind4 = self.index34()
        self.pos = np.zeros((n, 3))
        if len(ind3):
            f3 = self.faces[ind3, :3].astype(int)
            self.pos[ind3] = (self.verts[f3[:, 0]] + self.verts[f3[:, 1]] + self.verts[f3[:, 2]]) / 3.0
        if len(ind4):
            f4 = self.faces[ind4].astype(int)
            self.pos[ind4] = (self.verts[f4[:, 0]] + self.verts[f4[:, 1]] +
                              self.verts[f4[:, 2]] + self.verts[f4[:, 3]]) / 4.0
        tri, split = self._totriangles_flat()
        v1 = self.verts[tri[:, 0].astype(int)]
        v2 = self.verts[tri[:, 1].astype(int)]
        v3 = self.verts[tri[:, 2].astype(int)]
        vec1 = v1 - v2
        vec2 = v3 - v2
        nvec = np.cross(vec1, vec2)
        area = 0.5 * np.sqrt(np.sum(nvec * nvec, axis=1))
        vec1 = vec1 / np.maximum(np.sqrt(np.sum(vec1 * vec1, axis=1, keepdims=True)), 1e-14)
        nvec = nvec / np.maximum(np.sqrt(np.sum(nvec * nvec, axis=1, keepdims=True)), 1e-14)
        vec2 = np.cross(nvec, vec1)
        if len(split) == 0:
            self.area = area
            self.vec = [vec1, vec2, nvec]
            return
        self.area = area[:n].copy()
        np.add.at(self.area, split[:, 0], area[split[:, 1]])
        v1o, v2o, no = vec1[:n].copy(), vec2[:n].copy(), nvec[:n].copy()
        larger = area[split[:, 1]] > area[split[:, 0]]
        sel = split[larger]
        v1o[sel[:, 0]] = vec1[sel[:, 1]]
        v2o[sel[:, 0]] = vec2[sel[:, 1]]
        no[sel[:, 0]] = nvec[sel[:, 1]]
        self.vec = [v1o, v2o, no]

    def _norm_curv(self):
        """Centroids, areas and frames of curved elements (reference particle.py:551-614)."""
        n = self.nfaces
        _, w, _ = self.quad_integration()
        self.area = np.asarray(w.sum(axis=1)).ravel()
        ind3, ind4 = self.index34()
        tri = self.totriangles()[0]
        pos = np.zeros((n, 3))
        vec1 = np.zeros((n, 3))
        vec2 = np.zeros((n, 3))
        if len(ind3):
            c = np.array([-1, -1, -1, 4, 4, 4]) / 9
            cx = np.array([1, 0, -1, 4, -4, 0]) / 3
            cy = np.array([0, 1, -1, 4, 0, -4]) / 3
            vb = self.verts2[tri[ind3, :6].astype(int)]
            pos[ind3] = np.einsum("c,icd->id", c, vb)
            vec1[ind3] = np.einsum("c,icd->id", cy, vb)
            vec2[ind3] = np.einsum("c,icd->id", cx, vb)
        if len(ind4):
            fi = tri[ind4, :6].astype(int)
            pos[ind4] = self.verts2[fi[:, 5]]
            cx4 = np.array([1, 0, -1, 0, 0, 0])
            cy4 = np.array([0, -1, -1, 2, 2, -2])
            vb = self.verts2[fi]
            vec1[ind4] = np.einsum("c,icd->id", cy4, vb)
            vec2[ind4] = np.einsum("c,icd->id", cx4, vb)
        nvec = np.cross(vec1, vec2)
        nvec = nvec / np.maximum(np.linalg.norm(nvec, axis=1, keepdims=True), 1e-14)
        vec1 = vec1 / np.maximum(np.linalg.norm(vec1, axis=1, keepdims=True), 1e-14)
        vec2 = np.cross(nvec, vec1)
        self.pos = pos
        self.vec = [vec1, vec2, nvec]

    # ------------------------------------------------------- triangulation
    def _totriangles_flat(self, ind=None):
        """Split quads into (v0, v1, v2) + (v2, v3, v0) (reference particle.py:665-693)."""
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        _, ind4 = self.index34(ind)
        faces = self.faces[ind, :3].copy()
        if len(ind4):
            q = np.column_stack([self.faces[ind[ind4], 2], self.faces[ind[ind4], 3], self.faces[ind[ind4], 0]])
            faces = np.vstack([faces, q])
            split = np.column_stack([ind4, len(ind) + np.arange(len(ind4))])
        else:
            split = np.zeros((0, 2), dtype=int)
        return faces, split

    def _totriangles_curv(self, ind=None):
        """6-node triangles; quads give [0 1 2 e01 e12 c] + [2 3 0 e23 e30 c] (reference particle.py:695-725)."""
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        ind3, ind4 = self.index34(ind)
        faces = np.zeros((len(ind), 6))
        if len(ind3):
            faces[ind3] = self.faces2[ind[ind3]][:, [0, 1, 2, 4, 5, 6]]
        if len(ind4):
            faces[ind4] = self.faces2[ind[ind4]][:, [0, 1, 2, 4, 5, 8]]
            faces = np.vstack([faces, self.faces2[ind[ind4]][:, [2, 3, 0, 6, 7, 8]]])
            split = np.column_stack([ind4, len(ind) + np.arange(len(ind4))])
        else:
            split = np.zeros((0, 2), dtype=int)
        return faces, split

    def totriangles(self, ind=None):
        if self.interp == "flat":
            return self._totriangles_flat(ind)
        return self._totriangles_curv(ind)

    def _totriangles_plain(self, ind):
        """Quads split as (v0, v1, v2) + (v0, v2, v3) for flat quadrature (reference particle.py:1577-1604)."""
        faces = self.faces[ind]
        n = len(ind)
        isq = ~np.isnan(faces[:, 3])
        nq = int(np.sum(isq))
        if nq == 0:
            return faces[:, :3], np.zeros((0, 2), dtype=int)
        ft = np.zeros((n + nq, 3))
        ft[:n] = faces[:, :3]
        ft[n:, 0] = faces[isq, 0]
        ft[n:, 1] = faces[isq, 2]
        ft[n:, 2] = faces[isq, 3]
        return ft, np.column_stack([np.flatnonzero(isq), np.arange(n, n + nq)])

    # ---------------------------------------------------------- quadrature
    def quad_integration(self, ind=None):
        """28-point quadrature over faces ``ind``: (pos, w_csr (nind x npts), row)."""
        from scipy.sparse import csr_matrix
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        q = self.quad
        x, y, w = q.x, q.y, q.w
        m = len(w)
        if self.interp == "flat":
            ft, split = self._totriangles_plain(ind)
            ind3 = np.arange(len(ind))
            if len(split):
                ind3 = np.hstack([ind3, split[:, 0]])
            a = self.verts[ft[:, 1].astype(int)] - self.verts[ft[:, 0].astype(int)]
            b = self.verts[ft[:, 2].astype(int)] - self.verts[ft[:, 0].astype(int)]
            area = 0.5 * np.linalg.norm(np.cross(a, b), axis=1)
            shape = np.column_stack([x, y, 1 - x - y])
            vb = self.verts[ft[:, :3].astype(int)]
            pos = np.einsum("tc,icd->itd", shape, vb).reshape(-1, 3)
            weight = (w[None, :] * area[:, None]).ravel()
        else:
            ft, split = self._totriangles_curv(ind)
            ind3 = np.arange(len(ind))
            if len(split):
                ind3 = np.hstack([ind3, split[:, 0]])
            shape = tri6_shape(x, y)
            dx, dy = tri6_deriv(x, y)
            vb = self.verts2[ft[:, :6].astype(int)]
            pos = np.einsum("tc,icd->itd", shape, vb)
            px = np.einsum("tc,icd->itd", dx, vb)
            py = np.einsum("tc,icd->itd", dy, vb)
            jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
            pos = pos.reshape(-1, 3)
            weight = (0.5 * w[None, :] * jac).ravel()
        row = np.repeat(ind3, m)
        ntot = m * len(ind3)
        wsp = csr_matrix((weight, (row, np.arange(ntot))), shape=(len(ind), ntot))
        return pos, wsp, row

    def quadpol(self, ind=None):
        """Polar quadrature over faces ``ind``: (pos, weight, row) (reference particle.py:1276-1429)."""
        ind = np.arange(self.nfaces) if ind is None else np.asarray(ind)
        ind3, ind4 = self.index34(ind)
        q = self.quad
        m3, m4 = len(q.x3), len(q.x4)
        ntot = len(ind3) * m3 + len(ind4) * m4
        pos = np.zeros((ntot, 3))
        weight = np.zeros(ntot)
        row = np.zeros(ntot, dtype=int)
        off = 0
        if self.interp == "flat":
            if len(ind3):
                shape = np.column_stack([q.x3, q.y3, 1 - q.x3 - q.y3])
                vb = self.verts[self.faces[ind[ind3], :3].astype(int)]
                nb = len(ind3) * m3
                pos[off:off + nb] = np.einsum("tc,icd->itd", shape, vb).reshape(-1, 3)
                weight[off:off + nb] = (q.w3[None, :] * self.area[ind[ind3]][:, None]).ravel()
                row[off:off + nb] = np.repeat(ind3, m3)
                off += nb
            if len(ind4):
                shape = quad4_shape(q.x4, q.y4)
                dx, dy = quad4_deriv(q.x4, q.y4)
                vb = self.verts[self.faces[ind[ind4], :4].astype(int)]
                px = np.einsum("tc,icd->itd", dx, vb)
                py = np.einsum("tc,icd->itd", dy, vb)
                jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                nb = len(ind4) * m4
                pos[off:off + nb] = np.einsum("tc,icd->itd", shape, vb).reshape(-1, 3)
                weight[off:off + nb] = (q.w4[None, :] * jac).ravel()
                row[off:off + nb] = np.repeat(ind4, m4)
                off += nb
        else:
            faces = self.faces2[ind]
            if len(ind3):
                shape = tri6_shape(q.x3, q.y3)
                dx, dy = tri6_deriv(q.x3, q.y3)
                vb = self.verts2[faces[ind3][:, [0, 1, 2, 4, 5, 6]].astype(int)]
                px = np.einsum("tc,icd->itd", dx, vb)
                py = np.einsum("tc,icd->itd", dy, vb)
                jac = 0.5 * np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                nb = len(ind3) * m3
                pos[off:off + nb] = np.einsum("tc,icd->itd", shape, vb).reshape(-1, 3)
                weight[off:off + nb] = (q.w3[None, :] * jac).ravel()
                row[off:off + nb] = np.repeat(ind3, m3)
                off += nb
            if len(ind4):
                shape = quad9_shape(q.x4, q.y4)
                dx, dy = quad9_deriv(q.x4, q.y4)
                vb = self.verts2[faces[ind4][:, :9].astype(int)]
                px = np.einsum("tc,icd->itd", dx, vb)
                py = np.einsum("tc,icd->itd", dy, vb)
                jac = np.linalg.norm(np.cross(px, py, axis=2), axis=2)
                nb = len(ind4) * m4
                pos[off:off + nb] = np.einsum("tc,icd->itd", shape, vb).reshape(-1, 3)
                weight[off:off + nb] = (q.w4[None, :] * jac).ravel()
                row[off:off + nb] = np.repeat(ind4, m4)
                off += nb
        return pos, weight, row

    def bradius(self):
        """Radius of the smallest centroid-centred sphere enclosing each face's corners
        (reference particle.py:2848-2880)."""
        r = np.zeros(self.nfaces)
        ind3, ind4 = self.index34()
        for ind, nc in ((ind3, 3), (ind4, 4)):
            for i in range(nc):
                if len(ind):
                    vc = self.verts[self.faces[ind, i].astype(int)]
                    r[ind] = np.maximum(r[ind], np.linalg.norm(self.pos[ind] - vc, axis=1))
        return r

    # ------------------------------------------------------------- editing
    def shift(self, vec):
        vec = np.asarray(vec, dtype=float)
        self.verts = self.verts + vec
        if self.verts2 is not None:
            self.verts2 = self.verts2 + vec
        self._norm()
        return self

    def scale(self, s):
        s = np.asarray(s, dtype=float)
        self.verts = self.verts * s
        if self.verts2 is not None:
            self.verts2 = self.verts2 * s
        self._norm()
        return self

    def rot(self, angle, dir=None):
        """Rotate by ``angle`` degrees about the axis ``dir`` (default z): the
        vertices are multiplied from the right by expm(-angle K), K the
        cross-product matrix of the unit axis (reference particle.py:778-818)."""
        from scipy.linalg import expm
        d = np.array([0.0, 0.0, 1.0]) if dir is None else np.asarray(dir, dtype=float)
        d = d / np.linalg.norm(d)
        K = np.array([[0.0, -d[2], d[1]], [d[2], 0.0, -d[0]], [-d[1], d[0], 0.0]])
        R = expm(-(angle * np.pi / 180) * K)
        self.verts = self.verts @ R
        if self.verts2 is not None:
            self.verts2 = self.verts2 @ R
        self._norm()
        return self

    def flipfaces(self):
        """Reverse the orientation of every face (reference particle.py:868-908)."""
        new = copy.deepcopy(self)
        ind3, ind4 = new.index34()
        if len(ind3):
            new.faces[ind3, :3] = new.faces[ind3, :3][:, ::-1]
        if len(ind4):
            new.faces[ind4, :4] = new.faces[ind4, :4][:, ::-1]
        if new.faces2 is not None:
            if len(ind3):
                tmp = new.faces2[ind3][:, [2, 1, 0, 5, 4, 6]].copy()
                new.faces2[np.ix_(ind3, [0, 1, 2, 4, 5, 6])] = tmp
            if len(ind4):
                tmp = new.faces2[ind4][:, [3, 2, 1, 0, 6, 5, 4, 7]].copy()
                new.faces2[np.ix_(ind4, [0, 1, 2, 3, 4, 5, 6, 7])] = tmp
        new._norm()
        return new

    def flip(self, dir=0):
        """Mirror copy along the axes ``dir`` (0, 1, 2 or a list), faces
        reoriented so the normals stay outward (reference particle.py:843-866)."""
        new = copy.deepcopy(self)
        for d in ([dir] if np.isscalar(dir) else list(dir)):
            new.verts[:, d] = -new.verts[:, d]
            if new.verts2 is not None:
                new.verts2[:, d] = -new.verts2[:, d]
        return new.flipfaces()

    def clean(self, cutoff=1e-10):
        """Merge vertices equal to 8 decimals, turn quads with a repeated corner
        into triangles and drop faces of area <= cutoff * mean area
        (reference particle.py:2331-2395).

        As in the reference, the merged corner vertices take their rounded
        coordinates and the curved-node table (verts2, faces2) is left as it
        is; only the face selection touches it."""
        vr = mround(self.verts, 8)
        uniq, inv = np.unique(vr, axis=0, return_inverse=True)
        inv = inv.ravel()
        if len(uniq) != len(self.verts):
            f = self.faces.copy()
            ok = ~np.isnan(f)
            f[ok] = inv[f[ok].astype(int)]
            self.verts, self.faces = uniq, f
        for i in np.flatnonzero(~np.isnan(self.faces[:, 3])):
            v = self.faces[i, :4].astype(int)
            _, first = np.unique(v, return_index=True)
            if len(first) == 3:
                self.faces[i] = np.append(v[np.sort(first)], np.nan)
        self._norm()
        keep = np.flatnonzero(self.area > cutoff * np.mean(self.area))
        if len(keep) < self.nfaces:
            sel = self._compress(keep)
            self.verts, self.faces, self.verts2, self.faces2 = sel.verts, sel.faces, sel.verts2, sel.faces2
            self._norm()
        return self

    def select(self, index=None, carfun=None):
        """(selected, complement) particles by face index or by a predicate on
        the centroids (reference particle.py:910-962, index / carfun forms)."""
        if index is not None:
            idx = np.asarray(index, dtype=int)
        elif carfun is not None:
            idx = np.flatnonzero(carfun(self.pos[:, 0], self.pos[:, 1], self.pos[:, 2]))
        else:
            raise ValueError("select: give 'index' or 'carfun'")
        return self._compress(idx), self._compress(np.setdiff1d(np.arange(self.nfaces), idx))

    def _compress(self, idx):
        """Faces ``idx`` with unused vertices removed (reference particle.py:964-999)."""
        if len(idx) == 0:
            return Particle(np.zeros((0, 3)), np.zeros((0, 4)))

        def renumber(faces, verts):
            ok = ~np.isnan(faces)
            used = np.unique(faces[ok].astype(int))
            table = np.zeros(len(verts), dtype=int)
            table[used] = np.arange(len(used))
            faces = faces.copy()
            faces[ok] = table[faces[ok].astype(int)]
            return faces, verts[used]

        f, v = renumber(self.faces[idx], self.verts)
        new = Particle(v, f, interp=self.interp, norm=False)
        if self.verts2 is not None and self.faces2 is not None:
            new.faces2, new.verts2 = renumber(self.faces2[idx], self.verts2)
        new.quad = self.quad
        new._norm()
        return new

    def curved(self, key="flat"):
        if self.verts2 is None:
            self.midpoints()
        self.interp = "curv"
        self._norm()
        return self

    def flat(self):
        self.interp = "flat"
        self._norm()
        return self

    def midpoints(self):
        """Add flat edge midpoints (and quad centres) as curved-element nodes
        (reference particle.py:1775-1831, key 'flat')."""
        ind3, ind4 = self.index34()
        edges, face_edges = _edges(self.faces, ind3, ind4)
        nv = self.nverts
        mid = 0.5 * (self.verts[edges[:, 0]] + self.verts[edges[:, 1]])
        self.verts2 = np.vstack([self.verts, mid])
        self.faces2 = np.full((self.nfaces, 9), np.nan)
        self.faces2[:, :4] = self.faces
        if len(ind3):
            self.faces2[ind3, 4:7] = nv + face_edges[ind3, :3]
        if len(ind4):
            self.faces2[ind4, 4:8] = nv + face_edges[ind4, :4]
            f4 = self.faces[ind4].astype(int)
            cen = 0.25 * (self.verts[f4[:, 0]] + self.verts[f4[:, 1]] + self.verts[f4[:, 2]] + self.verts[f4[:, 3]])
            self.faces2[ind4, 8] = self.verts2.shape[0] + np.arange(len(ind4))
            self.verts2 = np.vstack([self.verts2, cen])
        return self

    def __add__(self, other):
        return self.vertcat(other)

    def vertcat(self, *others):
        """Concatenate particles (reference particle.py:1005-1044)."""
        v = self.verts.copy()
        f = self.faces.copy()
        v2 = None if self.verts2 is None else self.verts2.copy()
        f2 = None if self.faces2 is None else self.faces2.copy()
        for o in others:
            f = np.vstack([f, o.faces + v.shape[0]])
            v = np.vstack([v, o.verts])
            if v2 is not None and o.verts2 is not None:
                f2 = np.vstack([f2, o.faces2 + v2.shape[0]])
                v2 = np.vstack([v2, o.verts2])
        new = Particle(v, f, interp=self.interp, norm=False)
        new.verts2, new.faces2 = v2, f2
        new.quad = self.quad
        new._norm()
        return new

    # ------------------------------------------------------- device inputs
    def node_table(self):
        """Per-face curved nodes for the device quadrature kernels.

        Returns ``(nodes (n, 9, 3) float64, kind (n,) int32)`` where kind is
        0 = flat triangle (nodes 0..2), 1 = flat quad (0..3), 2 = curved
        triangle (nodes [v0 v1 v2 e01 e12 e20]), 3 = curved quad (nodes
        [v0 v1 v2 v3 e01 e12 e23 e30 centre]).
        """
        n = self.nfaces
        nodes = np.zeros((n, 9, 3))
        kind = np.zeros(n, dtype=np.int32)
        ind3, ind4 = self.index34()
        if self.interp == "flat":
            nodes[ind3, :3] = self.verts[self.faces[ind3, :3].astype(int)]
            nodes[ind4, :4] = self.verts[self.faces[ind4, :4].astype(int)]
            kind[ind4] = 1
        else:
            nodes[ind3, :6] = self.verts2[self.faces2[ind3][:, [0, 1, 2, 4, 5, 6]].astype(int)]
            nodes[ind4, :9] = self.verts2[self.faces2[ind4][:, :9].astype(int)]
            kind[ind3] = 2
            kind[ind4] = 3
        return nodes, kind

    def __repr__(self):
        return "Particle(nverts={}, nfaces={}, interp={!r})".format(self.nverts, self.nfaces, self.interp)


def _edges(faces, ind3, ind4):
    """Unique undirected edges and the edge index of each face side."""
    nf = len(faces)
    fe = np.full((nf, 4), -1, dtype=int)
    sides = []
    for ind, nc in ((ind3, 3), (ind4, 4)):
        if len(ind) == 0:
            continue
        f = faces[ind, :nc].astype(int)
        for k in range(nc):
            a, b = f[:, k], f[:, (k + 1) % nc]
            sides.append((ind, k, np.minimum(a, b), np.maximum(a, b)))
    if not sides:
        return np.zeros((0, 2), dtype=int), fe
    keys = np.concatenate([lo * (1 << 31) + hi for _, _, lo, hi in sides])
    uniq, inv = np.unique(keys, return_inverse=True)
    edges = np.column_stack([uniq >> 31, uniq & ((1 << 31) - 1)])
    off = 0
    for ind, k, lo, _ in sides:
        fe[ind, k] = inv[off:off + len(lo)]
        off += len(lo)
    return edges, fe


# ---------------------------------------------------------------------------
# shape generators
# ---------------------------------------------------------------------------

_SPHERE_SIZES = [32, 60, 144, 169, 225, 256, 289, 324, 361, 400, 441, 484,
                 529, 576, 625, 676, 729, 784, 841, 900, 961, 1024, 1225, 1444]
_sphere_cache = None


def _sphere_data():
    global _sphere_cache
    if _sphere_cache is None:
        _sphere_cache = dict(np.load(os.path.join(_DATA, "spheres.npz")))
    return _sphere_cache


def trisphere(n, diameter=1.0, **kwargs):
    """Triangulated sphere with curved (6-node) faces (reference mesh_generators.py:13-131).

    ``n`` is rounded to the nearest stored vertex count; the mesh has 2 n - 4
    faces.  Edge midpoints are projected onto the sphere.
    """
    if n is None or int(n) <= 0:
        raise ValueError("trisphere: 'n' must be a positive integer, got {!r}.".format(n))
    if not np.isfinite(diameter) or diameter <= 0:
        raise ValueError("trisphere: 'diameter' must be a positive finite float, got {!r}.".format(diameter))
    sizes = np.array(_SPHERE_SIZES)
    na = int(sizes[np.argmin(np.abs(sizes - int(n)))])
    d = _sphere_data()
    verts = 0.5 * d["verts{}".format(na)] * diameter
    faces = d["faces{}".format(na)].astype(float)
    p = Particle(verts, faces, norm=False)
    p.midpoints()
    v2 = p.verts2
    v2 = 0.5 * diameter * (v2 / np.linalg.norm(v2, axis=1, keepdims=True))
    kw = dict(kwargs)
    kw.setdefault("interp", "curv")
    return Particle(v2, p.faces2, **kw)


def mlinspace(a, b, n):
    """a + i (b - a) / (n - 1) with the last point exactly b: MATLAB's
    linspace, which differs from numpy's in the last bits
    (reference mnpbem/utils/matlab_compat.py:178-194)."""
    a, b, n = float(a), float(b), int(n)
    if n <= 0:
        return np.zeros(0)
    if n == 1:
        return np.array([b])
    y = a + np.arange(n, dtype=float) * (b - a) / (n - 1)
    y[-1] = b
    return y


def mround(x, digits=0):
    """Round half away from zero to ``digits`` decimals (MATLAB round;
    reference mnpbem/utils/matlab_compat.py:303-321)."""
    x = np.asarray(x, dtype=float)
    if digits == 0:
        return np.trunc(x + np.copysign(0.5, x))
    s = 10.0 ** digits
    return mround(x * s, 0) / s


def _fibonacci_sphere(n):
    """n points on the unit sphere along the golden-angle spiral
    (reference mesh_generators.py:341-370)."""
    t = np.arange(n, dtype=float) + 0.5
    lat = np.arccos(1 - 2 * t / n)
    lon = np.pi * (1 + 5 ** 0.5) * t
    p = np.column_stack([np.sin(lat) * np.cos(lon), np.sin(lat) * np.sin(lon), np.cos(lat)])
    return p / np.linalg.norm(p, axis=1, keepdims=True)


def _sphere_triangulate(verts):
    """Triangulate points on the unit sphere: rotate point 0 to the south pole,
    project the others stereographically onto z = 0, Delaunay-triangulate the
    plane (outward winding), and close the hole with a fan from point 0 over
    the convex hull (reference mesh_generators.py:373-443, MATLAB
    sphtriangulate)."""
    from scipy.spatial import ConvexHull, Delaunay
    c = verts[0]
    r3 = -c
    r2 = np.array([0.0, -r3[2], r3[1]]) if c[2] != 0 else np.array([-r3[1], r3[0], 0.0])
    r2 = r2 / np.linalg.norm(r2)
    rot = np.array([np.cross(r3, r2), r2, r3])
    vr = verts[1:] @ rot.T
    s = -1.0 / (vr[:, 2] + 1)
    plane = np.column_stack([vr[:, 0] * s, vr[:, 1] * s])
    tri = Delaunay(plane).simplices.copy()
    p3 = np.column_stack([plane, np.zeros(len(plane))])
    w = np.cross(p3[tri[:, 0]] - p3[tri[:, 1]], p3[tri[:, 2]] - p3[tri[:, 1]])
    up = w[:, 2] > 0
    tri[up] = tri[up][:, [0, 2, 1]]
    hull = ConvexHull(plane).vertices
    fan = np.column_stack([np.roll(hull, -1) + 1, hull + 1, np.zeros(len(hull), dtype=hull.dtype)])
    return np.vstack([tri + 1, fan])


def triellipsoid(n, axes):
    """Flat triangulated ellipsoid with about n vertices on a Fibonacci
    spiral, semi-axes ``axes`` (reference mesh_generators.py:446-473)."""
    v = _fibonacci_sphere(int(n))
    f = _sphere_triangulate(v)
    return Particle(v * np.asarray(axes, dtype=float), f)


def _surf2patch(x, y, z, triangles=False):
    """Faces and vertices of an (m, n) parametric grid, vertices in column-major
    order; quads [v00 v01 v11 v10] per cell, or all first triangles
    [v00 v01 v11] then all second ones [v00 v11 v10] (MATLAB surf2patch;
    reference mesh_generators.py:476-511)."""
    m, n = x.shape
    verts = np.column_stack([x.ravel(order="F"), y.ravel(order="F"), z.ravel(order="F")])
    i, j = np.meshgrid(np.arange(m - 1), np.arange(n - 1))
    i, j = i.ravel(), j.ravel()          # j outer, i inner
    v00, v10, v01, v11 = j * m + i, j * m + i + 1, (j + 1) * m + i, (j + 1) * m + i + 1
    if triangles:
        faces = np.vstack([np.column_stack([v00, v01, v11]), np.column_stack([v00, v11, v10])])
    else:
        faces = np.column_stack([v00, v01, v11, v10])
    return faces, verts


def fvgrid(x, y, triangles=False):
    """Curved-node table (verts2, faces2) of the flat grid x by y in the z = 0
    plane, faces in reversed surf2patch order (MATLAB fvgrid; reference
    mesh_generators.py:515-544)."""
    x, y = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
    if x.ndim == 1 and y.ndim == 1:
        x, y = np.meshgrid(x, y)
    faces, verts = _surf2patch(x, y, np.zeros_like(x), triangles)
    p = Particle(verts, faces[:, ::-1], norm=False)
    p.midpoints()
    return p.verts2, p.faces2


def trispheresegment(phi, theta, diameter=1.0, triangles=False, **kwargs):
    """Sphere segment over the (phi, theta) grid with curved nodes on the
    sphere (reference mesh_generators.py:549-585)."""
    ph, th = np.meshgrid(np.asarray(phi, dtype=float), np.asarray(theta, dtype=float))
    r = 0.5 * diameter
    faces, verts = _surf2patch(r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th), triangles)
    p = Particle(verts, faces).clean()
    p.midpoints()
    nrm = np.maximum(np.sqrt(np.sum(p.verts2 ** 2, axis=1, keepdims=True)), 1e-30)
    return Particle(r * (p.verts2 / nrm), p.faces2, **kwargs)


def trirod(diameter, height, n=None, triangles=False, **kwargs):
    """Rod (cylinder with hemispherical caps) along z: n = [nphi, ntheta, nz]
    grid points around, over each cap and along the cylinder
    (reference mesh_generators.py:592-640)."""
    nphi, ntheta, nz = [15, 20, 20] if n is None else list(n)
    phi = mlinspace(0, 2 * np.pi, nphi)
    theta = mlinspace(0, 0.5 * np.pi, ntheta)
    cap1 = trispheresegment(phi, theta, diameter, triangles=triangles, **kwargs)
    cap1.shift([0, 0, 0.5 * (height - diameter)])
    cap2 = cap1.flip(2)
    v2, f2 = fvgrid(phi, 0.5 * mlinspace(-1, 1, nz) * (height - diameter), triangles=triangles)
    r = 0.5 * diameter
    cyl = Particle(np.column_stack([r * np.cos(v2[:, 0]), r * np.sin(v2[:, 0]), v2[:, 1]]), f2, **kwargs)
    return (cap1 + cap2 + cyl).clean()


def tricube(n, length=1.0, e=0.25, **kwargs):
    """Cube with rounded edges: six n x n quad grids on the faces of the unit
    cube, graded with the exponent e, mapped onto the super-sphere
    |x|^(2/e) + ... and scaled to ``length`` (reference
    mesh_generators.py:643-702). It has 6 (n - 1)^2 quadrilateral faces."""
    length = np.asarray(length, dtype=float).ravel()
    length = np.full(3, length[0]) if length.size != 3 else length
    u = mlinspace(-0.5 ** e, 0.5 ** e, n)
    v2, faces = fvgrid(u, u)
    x = np.sign(v2[:, 0]) * np.abs(v2[:, 0]) ** (1.0 / e)
    y = np.sign(v2[:, 1]) * np.abs(v2[:, 1]) ** (1.0 / e)
    z = 0.5 * np.ones_like(x)
    sides = [(x, y, z), (y, x, -z), (y, z, x), (x, -z, y), (z, x, y), (-z, y, x)]
    parts = [Particle(np.column_stack(s), faces) for s in sides]
    p = parts[0].vertcat(*parts[1:]).clean()
    X, Y, Z = p.verts2[:, 0], p.verts2[:, 1], p.verts2[:, 2]
    az = np.arctan2(Y, X)
    el = np.arctan2(Z, np.sqrt(X ** 2 + Y ** 2))

    def spow_sin(a):
        return np.sign(np.sin(a)) * np.abs(np.sin(a)) ** e

    def spow_cos(a):
        return np.sign(np.cos(a)) * np.abs(np.cos(a)) ** e

    cube = np.column_stack([0.5 * spow_cos(el) * spow_cos(az), 0.5 * spow_cos(el) * spow_sin(az), 0.5 * spow_sin(el)])
    out = Particle(cube, p.faces2, **kwargs)
    return out.scale(length)


# ---------------------------------------------------------------------------
# compound particle
# ---------------------------------------------------------------------------


class ComParticle:
    """Particles with the dielectric media inside / outside each surface.

    ``ComParticle(eps, particles, inout, *closed, interp=...)`` where ``inout``
    rows are 1-based [inside, outside] indices into ``eps`` and ``closed``
    lists the particles forming closed surfaces (reference comparticle.py:59-128).
    """

    def __init__(self, eps, particles, inout, *closed_args, **kwargs):
        if eps is None or particles is None or inout is None:
            raise ValueError("ComParticle: eps, particles and inout are required")
        if len(eps) == 0:
            raise ValueError("ComParticle: 'eps' must contain at least one dielectric function.")
        self.eps = list(eps)
        if not isinstance(particles, (list, tuple)):
            particles = [particles]
        if "interp" in kwargs:
            for p in particles:
                if kwargs["interp"] == "curv":
                    p.curved()
                else:
                    p.flat()
        self.p = list(particles)
        io = np.atleast_2d(np.asarray(inout))
        if io.shape != (len(self.p), 2):
            raise ValueError("ComParticle: 'inout' must have shape (nparticles, 2); got {}".format(io.shape))
        if int(io.max()) > len(eps) or int(io.min()) < 1:
            raise ValueError("ComParticle: 'inout' indices out of range")
        self.inout = io.astype(int)
        self.closed = [None] * len(self.p)
        for arg in closed_args:
            idx = [arg] if np.isscalar(arg) else list(arg)
            for i in idx:
                if self.closed[abs(i) - 1] is None:
                    self.closed[abs(i) - 1] = list(idx)
        self._build()

    def _build(self):
        self.pc = self.p[0]
        for q in self.p[1:]:
            self.pc = self.pc + q
        self.nverts = sum(q.nverts for q in self.p)
        self.nfaces = sum(q.nfaces for q in self.p)
        self.np = len(self.p)

    @property
    def n(self):
        return self.nfaces

    @property
    def pos(self):
        return self.pc.pos

    @property
    def nvec(self):
        return self.pc.nvec

    @property
    def tvec1(self):
        return self.pc.tvec1

    @property
    def tvec2(self):
        return self.pc.tvec2

    @property
    def area(self):
        return self.pc.area

    @property
    def offsets(self):
        """Face offsets of the particles: particle i owns faces [off[i], off[i+1])."""
        return np.concatenate([[0], np.cumsum([q.nfaces for q in self.p])]).astype(np.int64)

    def index_func(self, i):
        """0-based face indices of 1-based particle(s) ``i``."""
        ii = [i] if np.isscalar(i) else list(i)
        off = self.offsets
        return np.concatenate([np.arange(off[k - 1], off[k]) for k in ii]).astype(int)

    @property
    def inout_faces(self):
        return np.repeat(self.inout, [q.nfaces for q in self.p], axis=0)

    def eps1(self, enei):
        return np.concatenate([np.full(q.nfaces, complex(np.asarray(self.eps[self.inout[i, 0] - 1](enei)[0]).flat[0]))
                               for i, q in enumerate(self.p)])

    def eps2(self, enei):
        return np.concatenate([np.full(q.nfaces, complex(np.asarray(self.eps[self.inout[i, 1] - 1](enei)[0]).flat[0]))
                               for i, q in enumerate(self.p)])

    def closed_particles(self):
        """For each particle i: the list of particle indices (0-based) forming
        its closed surface, or None.  Surfaces that need flipped faces are not
        supported by the device path.  When no particle was declared closed,
        every particle is taken as its own closed surface, as the reference
        does before its closed-surface correction (compgreen_ret.py:216-228)."""
        closed = self.closed
        if all(c is None for c in closed):
            closed = [[i + 1] for i in range(len(self.p))]
        out = []
        for i, c in enumerate(closed):
            if c is None:
                out.append(None)
                continue
            if any(int(x) < 0 for x in c):
                raise NotImplementedError("closed surfaces with flipped particles are not supported")
            out.append([int(x) - 1 for x in c])
        return out

    def bradius(self):
        return np.hstack([q.bradius() for q in self.p])

    # editing: applied to every particle, then the compound is rebuilt
    # (reference comparticle.py:420-487)
    def _each(self, method, *args, **kwargs):
        self.p = [getattr(q, method)(*args, **kwargs) for q in self.p]
        self._build()
        return self

    def shift(self, vec):
        return self._each("shift", vec)

    def scale(self, s):
        return self._each("scale", s)

    def rot(self, angle, dir=None):
        return self._each("rot", angle, dir)

    def flip(self, dir=0):
        return self._each("flip", dir)

    def flipfaces(self):
        return self._each("flipfaces")

    @property
    def verts(self):
        return self.pc.verts

    @property
    def faces(self):
        return self.pc.faces

    def ipart(self, ind):
        """(particle index, local face index) of global face indices
        (reference comparticle.py:987-1025)."""
        ind = np.atleast_1d(np.asarray(ind, dtype=int))
        off = self.offsets
        part = np.searchsorted(off, ind, side="right") - 1
        return part, ind - off[part]

    def __repr__(self):
        return "ComParticle(nparticles={}, nfaces={})".format(len(self.p), self.nfaces)
