"""Host-side case setup: node grids, the static geometry the step reads, and
initial states, in the reference's FieldBlock index space.

Every static field is computed with the reference's own formulas, as
vectorised numpy in the same per-element operation order:
  * cell centres (dual grid)       Block::calc_Dual_Grids      src/1_grid/1_MPCNS_Grid_GCL.cpp:6-21
  * face area vectors JD, Jac      compute_metric_fields       src/7_metric/Metric.cpp:108-326
  * |S|, |l*|, beta = |l*|/|S|     (faces)                     src/7_metric/Metric.cpp:398-474
  * |e|, |S*|, alpha = |e|/|S*|    (edges, dual-collapse cap)  src/7_metric/Metric.cpp:476-669
  * edge vectors dr                                             src/7_metric/Metric.cpp:1261-1328
  * B_cell / J_cell weights        SetupCellReconstructionWeights_
                                   Z4_Mercury/src/MercurySolver_ReconstructionSetup.cpp:29-193
  * neutral Na and photo rate      Initial_Na_And_PhotoRate_   Z4_Mercury/include/2_Initial.h:227-440
Ghost nodes of the periodic cube come from the analytic mapping (exact
periodic images); the reference fills ghost nodes that lie beyond two faces
at once by its own corner treatment, so static values in those ghost corners
differ — the step never reads them on a periodic block except through cell
centres of corner ghosts, which only the photo-rate and drag-shadow tests use.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

NGHOST = 4           # runtime ghost width (ngg)
NODE_GHOST = NGHOST + 1


@dataclass
class Arr:
    """A FieldBlock-style array: logical range [lo, hi), data[ni, nj, nk, nc]."""
    lo: tuple
    hi: tuple
    data: np.ndarray

    def sl(self, lo, hi):
        return tuple(slice(lo[a] - self.lo[a], hi[a] - self.lo[a]) for a in range(3))


def _view(a: np.ndarray, a_lo, lo, hi, di=0, dj=0, dk=0):
    """Sub-array of a node/cell array (logical origin a_lo) for logical
    range [lo, hi) shifted by (di, dj, dk)."""
    return a[lo[0] + di - a_lo[0]:hi[0] + di - a_lo[0],
             lo[1] + dj - a_lo[1]:hi[1] + dj - a_lo[1],
             lo[2] + dk - a_lo[2]:hi[2] + dk - a_lo[2]]


# ------------------------------------------------------------------ grids
def cube_nodes(n, amp: float = 0.05):
    """Nodes of the periodic curvilinear unit cube on [-G, n_a + 1 + G) per axis
    (n an int or three cell counts): x_a = xi_a + amp * sin(2 pi xi_b) * sin(2 pi xi_c),
    (a, b, c) cyclic, xi_a = index / n_a."""
    G = NODE_GHOST
    ns = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    idx = [np.arange(-G, m + 1 + G, dtype=np.float64) / m for m in ns]
    a, b, c = np.meshgrid(idx[0], idx[1], idx[2], indexing="ij")
    tp = 2.0 * math.pi
    x = a + amp * np.sin(tp * b) * np.sin(tp * c)
    y = b + amp * np.sin(tp * c) * np.sin(tp * a)
    z = c + amp * np.sin(tp * a) * np.sin(tp * b)
    return (-G, -G, -G), x, y, z


class Nodes:
    """Node coordinates of one block (with ghosts) and its dual points (cell
    centres): what the initial state needs, without the static fields."""

    def __init__(self, cells, node_lo, x, y, z, nghost: int = NGHOST):
        self.n = tuple(int(v) for v in cells)
        self.g = nghost
        self.nlo = node_lo
        self.x, self.y, self.z = x, y, z
        self.fields: dict[str, Arr] = {}
        self._dual()

    # helpers -------------------------------------------------------------
    def N(self, lo, hi, di=0, dj=0, dk=0):
        return tuple(_view(v, self.nlo, lo, hi, di, dj, dk) for v in (self.x, self.y, self.z))

    def D(self, lo, hi, di=0, dj=0, dk=0):
        return tuple(_view(v, self.dlo, lo, hi, di, dj, dk) for v in self.dual)

    def alloc_range(self, stag, g):
        return tuple(-g for _ in range(3)), tuple(self.n[a] + stag[a] + g for a in range(3))

    def _dual(self):
        g = self.g
        lo = (-g, -g, -g)
        hi = tuple(self.n[a] + g + 1 for a in range(3))
        out = []
        for X in (self.x, self.y, self.z):
            v = lambda di, dj, dk: _view(X, self.nlo, lo, hi, di, dj, dk)
            out.append(0.125 * (v(0, 0, 0) + v(-1, 0, 0) + v(0, -1, 0) + v(-1, -1, 0) +
                                v(0, 0, -1) + v(-1, 0, -1) + v(0, -1, -1) + v(-1, -1, -1)))
        self.dlo = lo
        self.dual = out
        # cell centre of cell (i, j, k) = dual(i + 1, j + 1, k + 1)
        clo = (-g - 1, -g - 1, -g - 1)
        chi = tuple(self.n[a] + g for a in range(3))
        for name, d in zip(("cell_x", "cell_y", "cell_z"), out):
            self.fields[name] = Arr(clo, chi, d[..., None].copy())

    def aos(self):
        """The nodes as one (ni, nj, nk, 3) array over the node range (the
        layout mhd_setup_geometry takes)."""
        return np.ascontiguousarray(np.stack([self.x, self.y, self.z], axis=-1))


class Geometry(Nodes):
    """Static fields of one block from its node coordinates (with ghosts)."""

    def __init__(self, cells, node_lo, x, y, z, nghost: int = NGHOST):
        super().__init__(cells, node_lo, x, y, z, nghost)
        self._faces()
        self._jac()
        self._face_hodge()
        self._edges()
        self._weights()

    def _faces(self):
        g = self.g
        specs = {  # (offsets of p_xp, p_yp, p_xyp) as in Metric.cpp:108-200
            "JDxi": ((1, 0, 0), ((0, 1, 0), (0, 0, 1), (0, 1, 1))),
            "JDet": ((0, 1, 0), ((0, 0, 1), (1, 0, 0), (1, 0, 1))),
            "JDze": ((0, 0, 1), ((1, 0, 0), (0, 1, 0), (1, 1, 0))),
        }
        for name, (stag, (oxp, oyp, oxyp)) in specs.items():
            lo, hi = self.alloc_range(stag, g)
            o = self.N(lo, hi)
            xp = self.N(lo, hi, *oxp)
            yp = self.N(lo, hi, *oyp)
            xyp = self.N(lo, hi, *oxyp)
            rx = [xp[a] - o[a] for a in range(3)]
            ry = [yp[a] - o[a] for a in range(3)]
            rx_ = [yp[a] - xyp[a] for a in range(3)]
            ry_ = [xp[a] - xyp[a] for a in range(3)]
            c1 = _cross(rx, ry)
            c2 = _cross(rx_, ry_)
            A = [c1[a] + c2[a] for a in range(3)]
            self.fields[name] = Arr(lo, hi, np.stack([0.5 * A[0], 0.5 * A[1], 0.5 * A[2]], axis=-1))

    def _jac(self):
        g = self.g - 1
        lo, hi = self.alloc_range((0, 0, 0), g)
        JX, JY, JZ = (self.fields[k] for k in ("JDxi", "JDet", "JDze"))
        xc = self.D(lo, hi, 1, 1, 1)

        def face(arr, d):
            return [arr.data[arr.sl(lo, hi) if d == 0 else _shift_sl(arr, lo, hi, d)][..., a] for a in range(3)]

        def fcen(nodes):
            return [0.25 * (nodes[0][a] + nodes[1][a] + nodes[2][a] + nodes[3][a]) for a in range(3)]

        N = self.N
        V = 0.0
        terms = [
            (face(JX, 0), -1, fcen([N(lo, hi), N(lo, hi, 0, 1, 0), N(lo, hi, 0, 0, 1), N(lo, hi, 0, 1, 1)])),
            (face(JX, 1), 1, fcen([N(lo, hi, 1, 0, 0), N(lo, hi, 1, 1, 0), N(lo, hi, 1, 0, 1), N(lo, hi, 1, 1, 1)])),
            (face(JY, 0), -1, fcen([N(lo, hi), N(lo, hi, 1, 0, 0), N(lo, hi, 0, 0, 1), N(lo, hi, 1, 0, 1)])),
            (face(JY, 2), 1, fcen([N(lo, hi, 0, 1, 0), N(lo, hi, 1, 1, 0), N(lo, hi, 0, 1, 1), N(lo, hi, 1, 1, 1)])),
            (face(JZ, 0), -1, fcen([N(lo, hi), N(lo, hi, 1, 0, 0), N(lo, hi, 0, 1, 0), N(lo, hi, 1, 1, 0)])),
            (face(JZ, 3), 1, fcen([N(lo, hi, 0, 0, 1), N(lo, hi, 1, 0, 1), N(lo, hi, 0, 1, 1), N(lo, hi, 1, 1, 1)])),
        ]
        V = np.zeros_like(xc[0])
        for Af, sgn, xf in terms:
            A = [(-Af[a] if sgn < 0 else Af[a]) for a in range(3)]
            d = [xf[a] - xc[a] for a in range(3)]
            V = V + (A[0] * d[0] + A[1] * d[1] + A[2] * d[2])
        self.fields["Jac"] = Arr(lo, hi, (V / 3.0)[..., None])

    def _face_hodge(self):
        g = self.g - 1
        eps = 1e-25
        for axis, (jd, an, bn) in enumerate((("JDxi", "Area_xi", "beta_xi"), ("JDet", "Area_eta", "beta_eta"),
                                             ("JDze", "Area_zeta", "beta_zeta"))):
            stag = tuple(1 if a == axis else 0 for a in range(3))
            lo, hi = self.alloc_range(stag, g)
            S = self.fields[jd].data[self.fields[jd].sl(lo, hi)]
            Smag = np.sqrt(S[..., 0] * S[..., 0] + S[..., 1] * S[..., 1] + S[..., 2] * S[..., 2])
            offL = [1, 1, 1]
            offL[axis] = 0
            cL = self.D(lo, hi, *offL)
            cR = self.D(lo, hi, 1, 1, 1)
            d = [cR[a] - cL[a] for a in range(3)]
            L = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
            with np.errstate(divide="ignore", invalid="ignore"):
                beta = np.where(Smag < eps, 0.0, L / Smag)
            self.fields[an] = Arr(lo, hi, Smag[..., None])
            self.fields[bn] = Arr(lo, hi, beta[..., None])

    def _edges(self):
        g = self.g - 1
        eps = 1e-25
        ratio, abs_tol = 1e-3, 1e-12
        # (edge offset, dual p00, p10, p01, p11 offsets)
        specs = [
            ((1, 0, 0), (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)),
            ((0, 1, 0), (0, 1, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1)),
            ((0, 0, 1), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)),
        ]
        names = (("dl_xi", "dr_xi", "alpha_xi"), ("dl_eta", "dr_eta", "alpha_eta"), ("dl_zeta", "dr_zeta", "alpha_zeta"))
        for axis, (eo, o00, o10, o01, o11) in enumerate(specs):
            stag = tuple(0 if a == axis else 1 for a in range(3))
            lo, hi = self.alloc_range(stag, g)
            r0 = self.N(lo, hi)
            r1 = self.N(lo, hi, *eo)
            dr = [r1[a] - r0[a] for a in range(3)]
            L = np.sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2])
            p00, p10, p01, p11 = (self.D(lo, hi, *o) for o in (o00, o10, o01, o11))
            a0 = _cross([p10[a] - p00[a] for a in range(3)], [p01[a] - p00[a] for a in range(3)])
            a1 = _cross([p01[a] - p11[a] for a in range(3)], [p10[a] - p11[a] for a in range(3)])
            Av = [0.5 * (a0[a] + a1[a]) for a in range(3)]
            Amag = np.sqrt(Av[0] * Av[0] + Av[1] * Av[1] + Av[2] * Av[2])
            with np.errstate(divide="ignore", invalid="ignore"):
                raw = np.where(Amag < eps, 0.0, L / Amag)

            def nrm(p, q):
                d = [q[a] - p[a] for a in range(3)]
                return np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])

            d00_10, d00_01, d10_11, d01_11 = nrm(p00, p10), nrm(p00, p01), nrm(p10, p11), nrm(p01, p11)
            d00_11, d10_01 = nrm(p00, p11), nrm(p10, p01)
            href = np.maximum(np.maximum(np.maximum(d00_10, d00_01), np.maximum(d10_11, d01_11)),
                              np.maximum(np.maximum(d00_11, d10_01), np.maximum(L, eps)))
            side_min = np.minimum(np.minimum(d00_10, d00_01), np.minimum(d10_11, d01_11))
            diag_min = np.minimum(d00_11, d10_01)
            touch = (L < abs_tol) | (side_min < ratio * href) | (diag_min < ratio * href) | (Amag < ratio * href * href)
            alpha = np.where(touch, 0.0, raw)
            dn, rn, an = names[axis]
            self.fields[dn] = Arr(lo, hi, L[..., None])
            self.fields[rn] = Arr(lo, hi, np.stack(dr, axis=-1))
            self.fields[an] = Arr(lo, hi, alpha[..., None])

    def _weights(self):
        g = self.g
        n = self.n
        lo, hi = (0, 0, 0), n
        WB = np.zeros(tuple(n[a] + 2 * g for a in range(3)) + (18,))
        WJ = np.zeros(tuple(n[a] + 2 * g for a in range(3)) + (36,))
        JX, JY, JZ = (self.fields[k] for k in ("JDxi", "JDet", "JDze"))
        s = np.empty(n + (6, 3))
        for a in range(3):
            s[..., 0, a] = -JX.data[JX.sl(lo, hi)][..., a]
            s[..., 1, a] = JX.data[_shift_sl(JX, lo, hi, 1)][..., a]
            s[..., 2, a] = -JY.data[JY.sl(lo, hi)][..., a]
            s[..., 3, a] = JY.data[_shift_sl(JY, lo, hi, 2)][..., a]
            s[..., 4, a] = -JZ.data[JZ.sl(lo, hi)][..., a]
            s[..., 5, a] = JZ.data[_shift_sl(JZ, lo, hi, 3)][..., a]
        N = self.N
        nodes8 = [N(lo, hi, *o) for o in ((0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1),
                                           (1, 1, 1))]
        xc = [0.125 * (nodes8[0][a] + nodes8[1][a] + nodes8[2][a] + nodes8[3][a] + nodes8[4][a] + nodes8[5][a] +
                       nodes8[6][a] + nodes8[7][a]) for a in range(3)]
        fsets = [((0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1)), ((1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)),
                 ((0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)), ((0, 1, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1)),
                 ((0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)), ((0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1))]
        smag = np.sqrt(s[..., 0] * s[..., 0] + s[..., 1] * s[..., 1] + s[..., 2] * s[..., 2])
        mu = np.empty(n + (6,))
        for q, fs in enumerate(fsets):
            pts = [N(lo, hi, *o) for o in fs]
            fc = [0.25 * (pts[0][a] + pts[1][a] + pts[2][a] + pts[3][a]) for a in range(3)]
            d = [fc[a] - xc[a] for a in range(3)]
            mu[..., q] = 1.0 / np.maximum(np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), 1.0e-14)
        sref = np.zeros(n)
        for q in range(6):
            sref = np.maximum(sref, smag[..., q])
        active = smag > 1.0e-10 * sref[..., None]
        M = np.zeros(n + (3, 3))
        for q in range(6):
            w = np.where(active[..., q], mu[..., q], 0.0)
            for a in range(3):
                for c in range(3):
                    M[..., a, c] = M[..., a, c] + np.where(active[..., q], w * s[..., q, a] * s[..., q, c], 0.0)
        Minv = _pinv_sym3(M)
        wb = np.zeros(n + (18,))
        for q in range(6):
            for a in range(3):
                val = mu[..., q] * (Minv[..., a, 0] * s[..., q, 0] + Minv[..., a, 1] * s[..., q, 1] +
                                    Minv[..., a, 2] * s[..., q, 2])
                wb[..., 6 * a + q] = np.where(active[..., q], val, 0.0)
        WB[g:g + n[0], g:g + n[1], g:g + n[2]] = wb
        # J_cell weights from the 12 edge vectors
        edges = [((0, 0, 0), (1, 0, 0)), ((0, 1, 0), (1, 1, 0)), ((0, 0, 1), (1, 0, 1)), ((0, 1, 1), (1, 1, 1)),
                 ((0, 0, 0), (0, 1, 0)), ((1, 0, 0), (1, 1, 0)), ((0, 0, 1), (0, 1, 1)), ((1, 0, 1), (1, 1, 1)),
                 ((0, 0, 0), (0, 0, 1)), ((1, 0, 0), (1, 0, 1)), ((0, 1, 0), (0, 1, 1)), ((1, 1, 0), (1, 1, 1))]
        l = np.empty(n + (12, 3))
        for q, (p0, p1) in enumerate(edges):
            a0, a1 = N(lo, hi, *p0), N(lo, hi, *p1)
            for a in range(3):
                l[..., q, a] = a1[a] - a0[a]
        ln = np.sqrt(l[..., 0] * l[..., 0] + l[..., 1] * l[..., 1] + l[..., 2] * l[..., 2])
        lmax = np.zeros(n)
        for q in range(12):
            lmax = np.maximum(lmax, ln[..., q])
        active = ln > 1.0e-10 * lmax[..., None]
        M = np.zeros(n + (3, 3))
        for q in range(12):
            for a in range(3):
                for c in range(3):
                    M[..., a, c] = M[..., a, c] + np.where(active[..., q], l[..., q, a] * l[..., q, c], 0.0)
        Minv = _pinv_sym3(M)
        wj = np.zeros(n + (36,))
        for q in range(12):
            for a in range(3):
                val = Minv[..., a, 0] * l[..., q, 0] + Minv[..., a, 1] * l[..., q, 1] + Minv[..., a, 2] * l[..., q, 2]
                wj[..., 12 * a + q] = np.where(active[..., q], val, 0.0)
        WJ[g:g + n[0], g:g + n[1], g:g + n[2]] = wj
        glo = (-g, -g, -g)
        ghi = tuple(n[a] + g for a in range(3))
        self.fields["Bcell_from_Bface_w"] = Arr(glo, ghi, WB)
        self.fields["Jcell_from_Jedge_w"] = Arr(glo, ghi, WJ)


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _shift_sl(arr: Arr, lo, hi, d):
    """Slice of ``arr`` for [lo, hi) shifted by +1 along axis d-1 (d in 1..3)."""
    sh = [0, 0, 0]
    sh[d - 1] = 1
    return tuple(slice(lo[a] + sh[a] - arr.lo[a], hi[a] + sh[a] - arr.lo[a]) for a in range(3))


def _pinv_sym3(M: np.ndarray) -> np.ndarray:
    """Pseudo-inverse of symmetric 3x3 matrices by cyclic Jacobi rotations
    (18 sweeps), dropping eigenvalues below 1e-10 of the largest — the
    eigen_sym3 / Minv construction of ReconstructionSetup.cpp:33-66,123-133.
    Works on component-major copies (A[p][q] contiguous over the cells)."""
    shp = M.shape[:-2]
    A = [[np.ascontiguousarray(M[..., p, q]) for q in range(3)] for p in range(3)]
    one, zero = np.ones(shp), np.zeros(shp)
    V = [[(one if a == c else zero).copy() for c in range(3)] for a in range(3)]
    for _ in range(18):
        for p in range(2):
            for q in range(p + 1, 3):
                apq = A[p][q]
                skip = np.abs(apq) <= 1.0e-16 * (np.abs(A[p][p]) + np.abs(A[q][q]) + 1.0)
                phi = 0.5 * np.arctan2(2.0 * apq, A[q][q] - A[p][p])
                c, s = np.cos(phi), np.sin(phi)
                c = np.where(skip, 1.0, c)
                s = np.where(skip, 0.0, s)
                app, aqq = A[p][p], A[q][q]
                r = 3 - p - q
                akp, akq = A[r][p], A[r][q]
                nkp = c * akp - s * akq
                nkq = s * akp + c * akq
                A[r][p] = np.where(skip, akp, nkp)
                A[p][r] = A[r][p]
                A[r][q] = np.where(skip, akq, nkq)
                A[q][r] = A[r][q]
                npp = c * c * app - 2.0 * s * c * apq + s * s * aqq
                nqq = s * s * app + 2.0 * s * c * apq + c * c * aqq
                A[p][p] = np.where(skip, app, npp)
                A[q][q] = np.where(skip, aqq, nqq)
                A[p][q] = np.where(skip, apq, 0.0)
                A[q][p] = A[p][q]
                for k in range(3):
                    vkp, vkq = V[k][p], V[k][q]
                    V[k][p] = np.where(skip, vkp, c * vkp - s * vkq)
                    V[k][q] = np.where(skip, vkq, s * vkp + c * vkq)
    lam = [A[0][0], A[1][1], A[2][2]]
    lmax = np.maximum(lam[0], np.maximum(lam[1], lam[2]))
    Minv = np.zeros(shp + (3, 3))
    for q in range(3):
        with np.errstate(divide="ignore"):
            inv = np.where(lam[q] > 1.0e-10 * lmax, 1.0 / lam[q], 0.0)
        for a in range(3):
            for c in range(3):
                Minv[..., a, c] = Minv[..., a, c] + V[a][q] * inv * V[c][q]
    Minv[lmax <= 1.0e-30] = 0.0
    return Minv


# ------------------------------------------------------------------ sources
def resistivity_eta(geom: Geometry, constants, eta_max: float = 1.25e7, r_inner: float = 0.84,
                    r_outer: float = 1.04, width: float = 0.02) -> dict:
    """Per-edge eta of the implicit resistive substep (ImplicitResistiveEtaAtEdge_,
    Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:222-258) on the owned
    edges, zero elsewhere: inver_Rem * window(r), r = |midpoint| of the edge,
    window = min(1, 0.5 (tanh((r - r_inner) / width) - tanh((r - r_outer) / width)))
    and 0 at or below 1e-10 (MercuryResistivityShape_,
    Z4_Mercury/src/physics/MercurySolver_Tools.cpp:50-69), inver_Rem = eta_max /
    (mu0 U_ref L_ref) (Tools.cpp:44); 0 on collapsed edges (|dl| <= 1e-12).
    Returns {"eta_res_xi" | "eta_res_eta" | "eta_res_zeta": Arr}."""
    inv_rem = eta_max / (constants.mu0 * constants.U_ref * constants.L_ref)
    out = {}
    for axis, name in enumerate(("eta_res_xi", "eta_res_eta", "eta_res_zeta")):
        stag = tuple(0 if a == axis else 1 for a in range(3))
        eo = tuple(1 if a == axis else 0 for a in range(3))
        lo, hi = geom.alloc_range(stag, geom.g)
        ilo, ihi = (0, 0, 0), tuple(geom.n[a] + stag[a] for a in range(3))
        p0, p1 = geom.N(ilo, ihi), geom.N(ilo, ihi, *eo)
        xm, ym, zm = (0.5 * (p0[a] + p1[a]) for a in range(3))
        r = np.sqrt(xm * xm + ym * ym + zm * zm)
        shape = 0.5 * (np.tanh((r - r_inner) / width) - np.tanh((r - r_outer) / width))
        shape = np.where(np.isfinite(shape) & (shape > 1e-10), np.minimum(1.0, shape), 0.0)
        dl = geom.fields[("dl_xi", "dl_eta", "dl_zeta")[axis]]
        dlv = dl.data[dl.sl(ilo, ihi)][..., 0]
        data = np.zeros(tuple(hi[a] - lo[a] for a in range(3)) + (1,))
        arr = Arr(lo, hi, data)
        data[arr.sl(ilo, ihi)] = np.where(np.abs(dlv) <= 1e-12, 0.0, inv_rem * shape)[..., None]
        out[name] = arr
    return out


def photo_rate(geom: Geometry, L_ref: float = 2.44e6):
    """Neutral Na [cm^-3] and Na+ production rate [cm^-3 s^-1] on the cell range
    [-g, n + g), Initial_Na_And_PhotoRate_ (Z4_Mercury/include/2_Initial.h:227-440)."""
    g = geom.g
    lo = (-g, -g, -g)
    hi = tuple(geom.n[a] + g for a in range(3))
    x, y, z = geom.D(lo, hi, 1, 1, 1)
    sk1, sk2 = 5.0e-5, 1.0e-5
    deg = math.acos(-1.0) / 180.0
    pi = math.acos(-1.0)
    r = np.sqrt(x * x + y * y + z * z)
    outside = (r > 1.0) & np.isfinite(r)
    rs = np.where(outside, r, 2.0)
    inv_r = 1.0 / rs
    rx, ry, rz = x * inv_r, y * inv_r, z * inv_r
    dr = L_ref * rs - L_ref
    r_factor = 1.0 / (rs * rs)

    def delta(lat, lon):
        clat = math.cos(lat)
        px, py, pz = clat * math.cos(lon), clat * math.sin(lon), math.sin(lat)
        return np.arccos(np.clip(rx * px + ry * py + rz * pz, -1.0, 1.0))

    def gauss2(d, H):
        a = d / H
        return np.exp(-(a * a))

    n_miv = 7.84e6 * np.exp(-dr / 431.0e3)
    n_td = 8.86e9 * np.exp(-dr / 100.0e3) * gauss2(delta(0.0, 0.0), 15.0 * deg)
    rad_psd = 4.06e10 * np.exp(-dr / 232.0e3)
    n_psd = rad_psd * (gauss2(delta(50.0 * deg, 0.0), 20.0 * deg) + gauss2(delta(-50.0 * deg, 0.0), 20.0 * deg))
    rad_sp = 5.67e6 * np.exp(-dr / 748.0e3)
    n_sp_day = rad_sp * (gauss2(delta(80.0 * deg, 0.0), 15.0 * deg) + gauss2(delta(-80.0 * deg, 0.0), 15.0 * deg))
    n_sp_night = rad_sp * (gauss2(delta(15.0 * deg, pi), 10.0 * deg) + gauss2(delta(-15.0 * deg, pi), 10.0 * deg))
    n_m3 = r_factor * (n_miv + n_td + n_psd + n_sp_day + n_sp_night)
    n_m3 = np.where(np.isfinite(n_m3) & (n_m3 >= 0.0), n_m3, 0.0)
    n_cm3 = np.where(outside, n_m3 * 1.0e-6, 0.0)
    shadow = (x < 0.0) & (np.sqrt(y * y + z * z) < 1.0)
    q = np.where(shadow, sk2, sk1) * n_cm3
    q = np.where(np.isfinite(q) & (q >= 0.0), q, 0.0)
    return Arr(lo, hi, n_cm3[..., None]), Arr(lo, hi, q[..., None])


# ------------------------------------------------------------------ initial state
def uniform_state(gamma=1.6667, NA=6.02e23, R_uni=8.314, U_ref=4.031e5, T_ref=1.7407e5, n_ref=4e7, M_ref=0.001,
                  ini=(4.03112887e5, 1.7407e5, 4e7, 0.001, 1.240347346e-1, 0.0), rho_small=None):
    """Uniform solar-wind states of both species as build_background_state
    builds them (Z4_Mercury/include/2_Initial.h:45-125).  The reference fills
    every allocated cell with them before any override, so they persist in
    ghost corners that no sync writes."""
    k_B = R_uni / NA
    rho_ref = M_ref / NA * n_ref
    U, T, n, Mm, c_y, c_z = ini
    rho0 = (n / n_ref) * (Mm / M_ref)
    c_x = -math.sqrt(1.0 - c_y * c_y - c_z * c_z)
    u0, v0, w0 = c_x * U / U_ref, c_y * U / U_ref, c_z * U / U_ref
    p0 = n * k_B * T / (rho_ref * U_ref * U_ref)
    qinf = np.array([rho0, rho0 * u0, rho0 * v0, rho0 * w0,
                     0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 / (gamma - 1.0)])
    if rho_small is None:
        rho_small = _reference_rho_small()
    pN = p0 * rho_small / 23.0
    qinfs = np.array([rho_small * rho0, 0.0, 0.0, 0.0, pN / (gamma - 1.0)])
    return qinf, qinfs


def _reference_rho_small():
    # Mercury_Initial's rho_small (Z4_Mercury/include/00_Mercury_Const.h)
    return 1e-6


class Uniform:
    """std::mt19937_64 with seed 20261203 + solve_id; uniforms (x >> 11) * 2^-53.
    Draws come from the library's host helper (mhd_seeded_uniform); the stream
    continues across calls."""

    def __init__(self, solve_id: int = 0):
        self.seed = 20261203 + solve_id
        self.used = 0

    def sym(self, a: float, count: int) -> np.ndarray:
        import ctypes

        from .capi import check, lib

        L = lib()
        L.mhd_seeded_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p]
        buf = np.empty(self.used + count)
        check(L.mhd_seeded_uniform(self.seed, self.used + count, a, buf.ctypes.data_as(ctypes.c_void_p)),
              "mhd_seeded_uniform")
        # the stream is regenerated from its start (the draws before this call
        # were produced with the same engine); amplitudes are per call
        out = buf[self.used:].copy()
        self.used += count
        return out


class _MT19937_64:
    """The 64-bit Mersenne Twister (Matsumoto & Nishimura, 2000), the engine
    std::mt19937_64 specifies."""
    NN, MM = 312, 156
    A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed: int):
        self.mt = [0] * self.NN
        self.mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, self.NN):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.mti = self.NN

    def next(self) -> int:
        if self.mti >= self.NN:
            mt = self.mt
            for i in range(self.NN):
                x = (mt[i] & self.UM) | (mt[(i + 1) % self.NN] & self.LM)
                xa = x >> 1
                if x & 1:
                    xa ^= self.A
                mt[i] = mt[(i + self.MM) % self.NN] ^ xa
            self.mti = 0
        x = self.mt[self.mti]
        self.mti += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & 0xFFFFFFFFFFFFFFFF


def host_uniform_sym(solve_id: int, a: float, count: int) -> np.ndarray:
    """The first ``count`` draws of Uniform(solve_id).sym(a, count), computed
    in Python with the engine above (no library call): for the few draws that
    size a workload, in processes that must not load the CUDA library."""
    g = _MT19937_64(20261203 + solve_id)
    out = np.empty(count)
    for q in range(count):
        out[q] = -a + 2.0 * a * ((g.next() >> 11) * 2.0 ** -53)
    return out


def orszag_tang_state(geom: Nodes, gamma: float = 1.6667, noise: float = 1e-3, solve_id: int = 0):
    """The cube case's initial state on a periodic cube: both ion fluids carry the
    Orszag-Tang vortex (rho = 1, p = 0.6, v = (-sin 2 pi y, sin 2 pi x, 0)) with
    multiplicative noise (1 + U[-noise, noise]) on every conserved component;
    B = curl A on the faces with A_z = (cos 4 pi x / (4 pi) + cos 2 pi y / (2 pi)) / sqrt(4 pi)
    line-integrated on the periodic edge set, each edge potential carrying the
    same multiplicative noise before the discrete curl (div B at roundoff).
    Draw order: cells (i, j, k lexicographic) x species (H, Na) x component,
    then xi, eta, zeta edges (i, j, k lexicographic).  Cells no sync writes
    (ghost corners) keep the uniform solar-wind state, as in the reference.
    Returns {name: Arr} for U_H, U_Na, B_xi, B_eta, B_zeta."""
    n = geom.n
    g = geom.g
    pi = math.acos(-1.0)
    rng = Uniform(solve_id)
    qinf, qinfs = uniform_state(gamma=gamma)
    shape = tuple(m + 2 * g for m in n)
    UH = np.empty(shape + (5,))
    UN = np.empty(shape + (5,))
    UH[...] = qinf
    UN[...] = qinfs
    xs, ys, _ = geom.D((0, 0, 0), n, 1, 1, 1)
    rho, p = 1.0, 0.6
    u = -np.sin(2.0 * pi * ys)
    v = np.sin(2.0 * pi * xs)
    w = np.zeros_like(u)
    q = np.stack([np.full_like(u, rho), rho * u, rho * v, rho * w,
                  p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)], axis=-1)
    ncell = n[0] * n[1] * n[2]
    own = tuple(slice(g, g + m) for m in n)
    nz = rng.sym(noise, ncell * 10).reshape(n + (2, 5))
    UH[own] = q * (1.0 + nz[:, :, :, 0, :])
    UN[own] = q * (1.0 + nz[:, :, :, 1, :])

    def Az(xx, yy):
        return (np.cos(4.0 * pi * xx) / (4.0 * pi) + np.cos(2.0 * pi * yy) / (2.0 * pi)) / math.sqrt(4.0 * pi)

    lo, hi = (0, 0, 0), n
    edges = []
    for off in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        a = geom.N(lo, hi)
        b = geom.N(lo, hi, *off)
        val = Az(0.5 * (a[0] + b[0]), 0.5 * (a[1] + b[1])) * (b[2] - a[2])
        edges.append(val * (1.0 + rng.sym(noise, ncell).reshape(n)))
    EX, EY, EZ = edges
    r = lambda A, di, dj, dk: np.roll(A, (-di, -dj, -dk), axis=(0, 1, 2))  # periodic shift: A[i+di]
    Bx = (EY - r(EY, 0, 0, 1)) + (r(EZ, 0, 1, 0) - EZ)
    By = (r(EX, 0, 0, 1) - EX) + (EZ - r(EZ, 1, 0, 0))
    Bz = (EX - r(EX, 0, 1, 0)) + (r(EY, 1, 0, 0) - EY)
    hi_c = tuple(m + g for m in n)
    out = {"U_H": Arr((-g,) * 3, hi_c, UH), "U_Na": Arr((-g,) * 3, hi_c, UN)}
    for name, Bv, ax in (("B_xi", Bx, 0), ("B_eta", By, 1), ("B_zeta", Bz, 2)):
        ext = [m + 2 * g for m in n]
        ext[ax] += 1
        arr = np.zeros(tuple(ext) + (1,))
        full = np.concatenate([Bv, Bv[(slice(0, 1) if ax == 0 else slice(None),
                                       slice(0, 1) if ax == 1 else slice(None),
                                       slice(0, 1) if ax == 2 else slice(None))]], axis=ax)
        sl = [slice(g, g + m) for m in n]
        sl[ax] = slice(g, g + n[ax] + 1)
        arr[tuple(sl)] = full[..., None]
        hi_ = list(hi_c)
        hi_[ax] += 1
        out[name] = Arr((-g,) * 3, tuple(hi_), arr)
    return out


def cube_case(n=32, amp: float = 0.05, solve_id: int = 0):
    """The periodic curvilinear cube case: geometry, sources and initial state of the cube
    (n cells per axis, or three per-axis counts for a periodic box).
    Returns (Geometry, {field name: Arr}) with every static input the step
    reads (reference names) and the initial state."""
    ns = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    lo, x, y, z = cube_nodes(ns, amp)
    geom = Geometry(ns, lo, x, y, z)
    f = dict(geom.fields)
    na, photo = photo_rate(geom)
    f["Na"] = na
    f["Photo_rate"] = photo
    g = NGHOST
    for name, ax in (("Badd_xi", 0), ("Badd_eta", 1), ("Badd_zeta", 2)):
        ext = [m + 2 * g for m in ns]
        ext[ax] += 1
        hi_ = [m + g for m in ns]
        hi_[ax] += 1
        f[name] = Arr((-g,) * 3, tuple(hi_), np.zeros(tuple(ext) + (1,)))
    for name, ax in (("taper_xi", 0), ("taper_eta", 1), ("taper_zeta", 2)):
        ext = [m + 1 + 2 * g for m in ns]
        ext[ax] -= 1
        t = np.zeros(tuple(ext) + (1,))
        sl = [slice(g, g + m + 1) for m in ns]
        sl[ax] = slice(g, g + ns[ax])
        t[tuple(sl)] = 1.0  # Hall taper with r_min = r_max = 0 is 1 everywhere it is read
        hi_ = [m + 1 + g for m in ns]
        hi_[ax] -= 1
        f[name] = Arr((-g,) * 3, tuple(hi_), t)
    f.update(orszag_tang_state(geom, solve_id=solve_id))
    return geom, f


def cube_state(n=32, amp: float = 0.05, solve_id: int = 0):
    """The periodic cube's nodes (AoS, for mhd_setup_geometry) and initial
    state only: the static fields are then computed on the device."""
    ns = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    lo, x, y, z = cube_nodes(ns, amp)
    nodes = Nodes(ns, lo, x, y, z)
    return nodes.aos(), orszag_tang_state(nodes, solve_id=solve_id)
