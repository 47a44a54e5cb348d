"""Synthetic icosahedral grid, metrics and fields for the tracer-advection path.

The reference reads its grid and metrics from binary snapshots (GRD_x, GRD_xt,
GMTR_* in dyn_horiz_adv_flux/src/main.f90:145-164) and ships no generator.
This module builds them:

* icosahedron split into the 10 diamonds of the reference's region table
  (kernels/NICAM/communication/src/mod_adm.f90:662-671: diamonds 1-5 have the
  north pole as corner N, 6-10 the south pole as corner S), each refined by
  recursive bisection of great-circle arcs to 2^glevel intervals per side
  (docs/NICAM/src/20_intro_nicam.tex:219-270), radius R = 6.371e6 m;
* cell positions GRD_x incl. halos (halos filled with the same COMM plan the
  kernels use, as NICAM fills them), triangle centres GRD_xt, arc midpoints
  GRD_xr, and the metrics GMTR_p (cell area), GMTR_t (triangle area and
  barycentric weights), GMTR_a (arc normals HN / tangents HT scaled by the
  arc length), with the pentagon and unused-triangle conventions of
  dyn_metrics/src/mod_gmtr.f90:46-741;
* gradient coefficients coef_grad with the stencil of
  dyn_metrics/src/mod_oprt.f90:499-734;
* the stretched vertical grid and the synthetic fields of the benchmark
  configurations (density, solid-body + noise winds, vertical mass flux,
  cosine-bell / slotted-cylinder / smooth random tracers).

All arrays use the reference layout written in C order (Fortran
var(gall,K0,lall,m) -> numpy shape (m, lall, gall)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

RADIUS = 6.371e6
TI, TJ = 0, 1
AI, AIJ, AJ = 0, 1, 2


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _tri_area(a, b, c):
    """Solid angle of spherical triangles with unit-vector corners (Van Oosterom & Strackee)."""
    num = np.abs(np.einsum("...i,...i", a, np.cross(b, c)))
    den = 1.0 + np.einsum("...i,...i", a, b) + np.einsum("...i,...i", b, c) + np.einsum("...i,...i", c, a)
    return 2.0 * np.arctan2(num, den)


def _arc_angle(a, b):
    """Angle between unit vectors, robust for small angles."""
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=-1), np.einsum("...i,...i", a, b))


def apply_plan_numpy(plan, var, var_pl):
    """Host-side application of a composed halo plan (dst[e] <- src[e] over the flat point
    index: region points, then the 12 pole slots) to var (m, lall, K, gall), var_pl (m, 2, K, 6)."""
    dst, src = plan
    m, L, K, G = var.shape
    flat = np.concatenate([var.transpose(0, 2, 1, 3).reshape(m, K, L * G),
                           var_pl.transpose(0, 2, 1, 3).reshape(m, K, 12)], axis=2)
    flat[:, :, dst] = flat[:, :, src]
    var[...] = flat[:, :, :L * G].reshape(m, K, L, G).transpose(0, 2, 1, 3)
    var_pl[...] = flat[:, :, L * G:].reshape(m, K, 2, 6).transpose(0, 2, 1, 3)


def diamond_corners():
    """Corners (W, S, E, N) of the 10 diamonds as unit vectors, shape (10, 4, 3)."""
    lat = math.atan(0.5)
    up = [np.array([math.cos(lat) * math.cos(math.radians(72 * k)), math.cos(lat) * math.sin(math.radians(72 * k)),
                    math.sin(lat)]) for k in range(5)]
    lo = [np.array([math.cos(lat) * math.cos(math.radians(72 * k + 36)),
                    math.cos(lat) * math.sin(math.radians(72 * k + 36)), -math.sin(lat)]) for k in range(5)]
    npole, spole = np.array([0.0, 0.0, 1.0]), np.array([0.0, 0.0, -1.0])
    corners = np.zeros((10, 4, 3))
    for k in range(5):  # northern diamond k+1: W = U_k, S = L_k, E = U_k+1, N = north pole
        corners[k] = [up[k], lo[k], up[(k + 1) % 5], npole]
    for k in range(5):  # southern diamond under U_k: W = L_k-1, S = south pole, E = L_k, N = U_k
        d = 5 if k == 0 else 10 - k
        corners[d] = [lo[(k - 1) % 5], spole, lo[k], up[k]]
    return corners


def diamond_lattice(glevel):
    """Points of the 10 diamonds, shape (10, N+1, N+1, 3) indexed [d, a, b] with a along W->S,
    b along W->N, N = 2^glevel; recursive bisection with normalised great-circle midpoints."""
    n = 1 << glevel
    x = np.zeros((10, n + 1, n + 1, 3))
    c = diamond_corners()
    x[:, 0, 0], x[:, n, 0], x[:, n, n], x[:, 0, n] = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    h = n
    while h > 1:
        g = h // 2
        # midpoints along a, along b, and along the a=b diagonal of every coarse cell
        x[:, g:n:h, 0:n + 1:h] = _unit(x[:, 0:n - g:h, 0:n + 1:h] + x[:, h:n + 1:h, 0:n + 1:h])
        x[:, 0:n + 1:h, g:n:h] = _unit(x[:, 0:n + 1:h, 0:n - g:h] + x[:, 0:n + 1:h, h:n + 1:h])
        x[:, g:n:h, g:n:h] = _unit(x[:, 0:n - g:h, 0:n - g:h] + x[:, h:n + 1:h, h:n + 1:h])
        h = g
    return x


def vertical_grid(kall, ztop=40.0e3, stretch=1.5):
    """Stretched heights: half levels z_h(k) = ztop*((k-kmin)/(kmax-kmin+1))^stretch for
    k = kmin..kmax+1 (1-based), full levels at mid-layer, one ghost level each side.
    Returns dict of arrays of length kall (0-based index = Fortran k-1)."""
    kmin, kmax = 2, kall - 1
    nl = kmax - kmin + 1
    zh = np.zeros(kall)
    for k in range(kmin, kmax + 2):
        zh[k - 1] = ztop * ((k - kmin) / nl) ** stretch
    z = np.zeros(kall)
    for k in range(kmin, kmax + 1):
        z[k - 1] = 0.5 * (zh[k - 1] + zh[k])
    z[kmin - 2] = -z[kmin - 1]
    z[kall - 1] = 2 * ztop - z[kmax - 1]
    dz = np.zeros(kall)
    for k in range(kmin, kmax + 1):
        dz[k - 1] = zh[k] - zh[k - 1]
    dz[0], dz[kall - 1] = dz[kmin - 1], dz[kmax - 1]
    afact = np.zeros(kall)
    for k in range(kmin, kall):  # face k (between k-1 and k): linear interpolation in height
        afact[k - 1] = (zh[k - 1] - z[k - 2]) / (z[k - 1] - z[k - 2])
    afact[0] = 1.0
    bfact = 1.0 - afact
    return dict(z=z, zh=zh, rdgz=1.0 / dz, afact=afact, bfact=bfact, dz=dz, kmin=kmin, kmax=kmax)


@dataclass
class Grid:
    glevel: int
    rlevel: int
    kall: int
    R: float = RADIUS
    arrays: dict = field(default_factory=dict)
    # provider of the region topology and the halo plan: an object with
    # topology_info(glevel, rlevel) -> (have_sgp, rgn4pl, pole_ring) and
    # comm_plan(glevel, rlevel, pole_fill) -> (dst, src); None: this library's host tables
    tables: object = None

    def __post_init__(self):
        gl, rl = self.glevel, self.rlevel
        self.nmax = 1 << (gl - rl)
        self.gall_1d = self.nmax + 2
        self.gall = self.gall_1d ** 2
        self.gmin, self.gmax = 2, self.nmax + 1
        self.lall = 10 * 4 ** rl
        self.kmin, self.kmax = (2, self.kall - 1) if self.kall > 1 else (1, 1)
        tables = self.tables
        if tables is None:
            from . import api as tables
        self.have_sgp, self.rgn4pl, self.pole_ring = tables.topology_info(gl, rl)
        self.plan = tables.comm_plan(gl, rl, False)
        self.tables = None  # the plan is held; the provider is not needed after construction
        self._build_positions()
        self._build_metrics()
        self._build_gradient()
        self.arrays.update({k: np.ascontiguousarray(v) for k, v in vertical_grid(self.kall).items()
                            if isinstance(v, np.ndarray)})

    # -- helpers on (m, lall, G, G) views, index [.., l, j-1, i-1]
    def _fill_halo(self, a, a_pl):
        """Halo fill of per-column arrays a (m, lall, gall) / a_pl (m, 2, 6) with the COMM plan."""
        m = a.shape[0]
        v = a.reshape(m, self.lall, 1, self.gall).copy()
        vp = a_pl.reshape(m, 2, 1, 6).copy()
        apply_plan_numpy(self.plan, v, vp)
        return v.reshape(a.shape), vp.reshape(a_pl.shape)

    def _build_positions(self):
        gl, rl, G, n = self.glevel, self.rlevel, self.gall_1d, self.nmax
        lat = diamond_lattice(gl)
        rl1 = 1 << rl
        x = np.zeros((3, self.lall, G, G))
        ii = np.arange(self.gmin, self.gmax + 1)
        for r in range(self.lall):
            d, rem = divmod(r, rl1 * rl1)
            jr, ir = divmod(rem, rl1)
            a = ir * n + (ii - self.gmin)
            b = jr * n + (ii - self.gmin)
            blk = lat[d][np.ix_(a, b)]  # [a, b, 3] = [i, j, 3]
            x[:, r, self.gmin - 1:self.gmax, self.gmin - 1:self.gmax] = blk.transpose(2, 1, 0)
        xp = np.zeros((3, 2, 6))
        xp[:, 0, 0] = [0, 0, 1.0]
        xp[:, 1, 0] = [0, 0, -1.0]
        xf, xpf = self._fill_halo(x.reshape(3, self.lall, self.gall), xp)
        self.xu = xf.reshape(3, self.lall, G, G)  # unit vectors
        self.xpu = xpf
        A = self.arrays
        A["GRD_x"] = np.ascontiguousarray(xf * self.R)
        A["GRD_x_pl"] = np.ascontiguousarray(xpf * self.R)

    def _build_metrics(self):
        R, G, L = self.R, self.gall_1d, self.lall
        g0, g1 = self.gmin - 1, self.gmax - 1  # 0-based gmin, gmax
        X = np.moveaxis(self.xu, 0, -1)  # (L, G(j), G(i), 3)
        # triangle centres (unit) for (i,j) in [gmin-1, gmax]^2; TI=(ij,ip1j,ip1jp1), TJ=(ij,ip1jp1,ijp1)
        s = slice(g0 - 1, g1 + 1)
        sp = slice(g0, g1 + 2)
        v_ij, v_ip1j, v_ip1jp1, v_ijp1 = X[:, s, s], X[:, s, sp], X[:, sp, sp], X[:, sp, s]
        xt = np.zeros((2, L, G, G, 3))
        xt[TI][:, s, s] = _unit(v_ij + v_ip1j + v_ip1jp1)
        xt[TJ][:, s, s] = _unit(v_ij + v_ip1jp1 + v_ijp1)
        verts = {TI: (v_ij, v_ip1j, v_ip1jp1), TJ: (v_ij, v_ip1jp1, v_ijp1)}
        gt = np.zeros((5, 2, L, G, G))
        for t in (TI, TJ):
            c = xt[t][:, s, s]
            a1 = _tri_area(c, verts[t][1], verts[t][2])
            a2 = _tri_area(c, verts[t][2], verts[t][0])
            a3 = _tri_area(c, verts[t][0], verts[t][1])
            area = a1 + a2 + a3
            with np.errstate(divide="ignore", invalid="ignore"):
                gt[0, t][:, s, s] = area * R * R
                gt[1, t][:, s, s] = 1.0 / (area * R * R)
                gt[2, t][:, s, s] = a1 / area
                gt[3, t][:, s, s] = a2 / area
                gt[4, t][:, s, s] = a3 / area
        # unused triangles and the pentagon (mod_gmtr.f90:293-299)
        gt[:, TI, :, g0 - 1, g1] = gt[:, TJ, :, g0 - 1, g1]
        xt[TI][:, g0 - 1, g1] = xt[TJ][:, g0 - 1, g1]
        gt[:, TJ, :, g1, g0 - 1] = gt[:, TI, :, g1, g0 - 1]
        xt[TJ][:, g1, g0 - 1] = xt[TI][:, g1, g0 - 1]
        sg = np.nonzero(self.have_sgp)[0]
        gt[:, TI, sg, g0 - 1, g0 - 1] = gt[:, TJ, sg, g0 - 1, g0]
        xt[TI][sg, g0 - 1, g0 - 1] = xt[TJ][sg, g0 - 1, g0]
        self.xt = xt
        # hexagon arcs (mod_gmtr.f90:566-676): AI from xt(ij,TI) to xt(ijm1,TJ),
        # AIJ from xt(ij,TJ) to xt(ij,TI), AJ from xt(im1j,TI) to xt(ij,TJ)
        ga = np.zeros((12, 3, L, G, G))
        xr = np.zeros((3, 3, L, G, G))
        fr = np.zeros((3, L, G, G, 3))
        to = np.zeros((3, L, G, G, 3))
        fr[AI][:, g0:g1 + 1, g0 - 1:g1 + 1] = xt[TI][:, g0:g1 + 1, g0 - 1:g1 + 1]
        to[AI][:, g0:g1 + 1, g0 - 1:g1 + 1] = xt[TJ][:, g0 - 1:g1, g0 - 1:g1 + 1]
        fr[AIJ][:, s, s] = xt[TJ][:, s, s]
        to[AIJ][:, s, s] = xt[TI][:, s, s]
        # unused hexagon arcs (mod_gmtr.f90:612-616)
        fr[AIJ][:, g0 - 1, g1] = xt[TJ][:, g0 - 1, g1]
        to[AIJ][:, g0 - 1, g1] = xt[TI][:, g0, g1]
        fr[AIJ][:, g1, g0 - 1] = xt[TJ][:, g1, g0]
        to[AIJ][:, g1, g0 - 1] = xt[TI][:, g1, g0 - 1]
        fr[AJ][:, g0 - 1:g1 + 1, g0:g1 + 1] = xt[TI][:, g0 - 1:g1 + 1, g0 - 1:g1]
        to[AJ][:, g0 - 1:g1 + 1, g0:g1 + 1] = xt[TJ][:, g0 - 1:g1 + 1, g0:g1 + 1]
        fr[AJ][sg, g0 - 1, g0] = xt[TI][sg, g0, g0]  # pentagon (mod_gmtr.f90:650-653)
        to[AJ][sg, g0 - 1, g0] = xt[TJ][sg, g0 - 1, g0]
        for a in (AI, AIJ, AJ):
            f, t = fr[a], to[a]
            ok = (np.linalg.norm(f, axis=-1) > 0) & (np.linalg.norm(t, axis=-1) > 0)
            dist = _arc_angle(np.where(ok[..., None], f, 1), np.where(ok[..., None], t, 1)) * R
            nv = np.cross(f, t)
            nl = np.linalg.norm(nv, axis=-1)
            tv = t - f
            tl = np.linalg.norm(tv, axis=-1)
            with np.errstate(divide="ignore", invalid="ignore"):
                hn = np.where((ok & (nl > 0))[..., None], nv * (dist / nl)[..., None], 0.0)
                ht = np.where((ok & (tl > 0))[..., None], tv * (dist / tl)[..., None], 0.0)
            for x in range(3):
                ga[0 + x, a] = hn[..., x]
                ga[3 + x, a] = ht[..., x]
            mid = np.where(ok[..., None], _unit(np.where(ok[..., None], f + t, 1)), 0.0) * R
            for x in range(3):
                xr[x, a] = mid[..., x]
        # cell areas (mod_gmtr.f90:101-152): 6 triangles around the cell, centre GRD_x
        si = slice(g0, g1 + 1)
        sm = slice(g0 - 1, g1)
        w = [xt[TJ][:, sm, si], xt[TI][:, si, si], xt[TJ][:, si, si], xt[TI][:, si, sm], xt[TJ][:, sm, sm],
             xt[TI][:, sm, sm]]
        w = [wk.copy() for wk in w]
        w[5][sg, 0, 0] = w[0][sg, 0, 0]  # pentagon: vertex 6 = vertex 1
        w.append(w[0])
        c0 = X[:, si, si]
        area = sum(_tri_area(c0, w[v], w[v + 1]) for v in range(6)) * R * R
        gp = np.zeros((8, L, G, G))
        gp[0][:, si, si] = area
        gp[1][:, si, si] = 1.0 / area
        lon = np.arctan2(X[..., 1], X[..., 0])
        gp[2] = -np.sin(lon)
        gp[3] = np.cos(lon)
        gp[5] = -X[..., 2] * np.cos(lon)
        gp[6] = -X[..., 2] * np.sin(lon)
        gp[7] = X[..., 0] * np.cos(lon) + X[..., 1] * np.sin(lon)
        # ---- poles
        xpu = np.moveaxis(self.xpu, 0, -1)  # (2, 6, 3)
        xt_pl = np.zeros((2, 6, 3))
        gt_pl = np.zeros((5, 2, 6))
        ga_pl = np.zeros((18, 2, 6))
        xr_pl = np.zeros((3, 2, 6))
        gp_pl = np.zeros((8, 2, 6))
        for p in range(2):
            for v in range(2, 7):
                vp = 2 if v == 6 else v + 1
                xt_pl[p, v - 1] = _unit(xpu[p, 0] + xpu[p, v - 1] + xpu[p, vp - 1])
            for v in range(2, 7):
                vp = 2 if v == 6 else v + 1
                c = xt_pl[p, v - 1]
                a1 = _tri_area(c, xpu[p, v - 1], xpu[p, vp - 1])
                a2 = _tri_area(c, xpu[p, vp - 1], xpu[p, 0])
                a3 = _tri_area(c, xpu[p, 0], xpu[p, v - 1])
                ar = a1 + a2 + a3
                gt_pl[:, p, v - 1] = [ar * R * R, 1 / (ar * R * R), a1 / ar, a2 / ar, a3 / ar]
            for v in range(2, 7):
                vm = 6 if v == 2 else v - 1
                f, t = xt_pl[p, vm - 1], xt_pl[p, v - 1]
                dist = _arc_angle(f, t) * R
                nv = np.cross(f, t)
                ga_pl[0:3, p, v - 1] = nv * dist / np.linalg.norm(nv)
                ga_pl[3:6, p, v - 1] = (t - f) * dist / np.linalg.norm(t - f)
                xr_pl[:, p, v - 1] = _unit(f + t) * R
            area = sum(_tri_area(xpu[p, 0], xt_pl[p, v - 1], xt_pl[p, (2 if v == 6 else v + 1) - 1])
                       for v in range(2, 7)) * R * R
            gp_pl[0, p, 0] = area
            gp_pl[1, p, 0] = 1.0 / area
        # halo areas come from the neighbour regions and the poles, as after a COMM of GMTR_p
        gpf, _ = self._fill_halo(gp.reshape(8, L, self.gall), gp_pl)
        A = self.arrays
        A["GRD_xt"] = np.ascontiguousarray(np.moveaxis(xt, -1, 0).reshape(3, 2, L, self.gall) * R)
        A["GRD_xt_pl"] = np.ascontiguousarray(np.moveaxis(xt_pl, -1, 0) * R)
        A["GRD_xr"] = np.ascontiguousarray(xr.reshape(3, 3, L, self.gall))
        A["GRD_xr_pl"] = np.ascontiguousarray(xr_pl)
        A["GMTR_p"] = np.ascontiguousarray(gpf)
        A["GMTR_p_pl"] = np.ascontiguousarray(gp_pl)
        A["GMTR_t"] = np.ascontiguousarray(gt.reshape(5, 2, L, self.gall))
        A["GMTR_t_pl"] = np.ascontiguousarray(gt_pl)
        A["GMTR_a"] = np.ascontiguousarray(ga.reshape(12, 3, L, self.gall))
        A["GMTR_a_pl"] = np.ascontiguousarray(ga_pl)

    def _build_gradient(self):
        """coef_grad(gall,0:6,3,lall) -> shape (lall, 3, 7, gall); the stencil of
        OPRT_gradient_setup (dyn_metrics/src/mod_oprt.f90:499-734), neighbour order
        ij, ip1j, ip1jp1, ijp1, im1j, im1jm1, ijm1."""
        A = self.arrays
        L, G, gall = self.lall, self.gall_1d, self.gall
        gt = A["GMTR_t"].reshape(5, 2, L, gall)
        ga = A["GMTR_a"].reshape(12, 3, L, gall)
        rarea = A["GMTR_p"][1]
        cg = np.zeros((L, 3, 7, gall))
        jj, ii = np.meshgrid(np.arange(self.gmin, self.gmax + 1), np.arange(self.gmin, self.gmax + 1), indexing="ij")
        ij = ((jj - 1) * G + ii - 1).ravel()
        im1j, im1jm1, ijm1 = ij - 1, ij - G - 1, ij - G
        W1, W2, W3 = 2, 3, 4

        def T(c, t, w):
            return gt[w, t][:, c]

        for d in range(3):
            def Aa(c, a):
                return ga[d, a][:, c]

            f = 0.5 * rarea[:, ij]
            c0 = (T(ij, TI, W1) * Aa(ij, AI) + T(ij, TI, W1) * Aa(ij, AIJ) + T(ij, TJ, W1) * Aa(ij, AIJ)
                  + T(ij, TJ, W1) * Aa(ij, AJ) + T(im1j, TI, W2) * Aa(ij, AJ) - T(im1j, TI, W2) * Aa(im1j, AI)
                  - T(im1jm1, TJ, W2) * Aa(im1j, AI) - T(im1jm1, TI, W3) * Aa(im1jm1, AIJ)
                  - T(im1jm1, TJ, W2) * Aa(im1jm1, AIJ) - T(im1jm1, TI, W3) * Aa(ijm1, AJ)
                  - T(ijm1, TJ, W3) * Aa(ijm1, AJ) + T(ijm1, TJ, W3) * Aa(ij, AI)
                  - 2 * Aa(ij, AIJ) - 2 * Aa(ij, AJ) + 2 * Aa(im1j, AI) + 2 * Aa(im1jm1, AIJ)
                  + 2 * Aa(ijm1, AJ) - 2 * Aa(ij, AI)) * f
            c1 = (-T(ijm1, TJ, W2) * Aa(ijm1, AJ) + T(ijm1, TJ, W2) * Aa(ij, AI) + T(ij, TI, W2) * Aa(ij, AI)
                  + T(ij, TI, W2) * Aa(ij, AIJ)) * f
            c2 = (T(ij, TI, W3) * Aa(ij, AI) + T(ij, TI, W3) * Aa(ij, AIJ) + T(ij, TJ, W2) * Aa(ij, AIJ)
                  + T(ij, TJ, W2) * Aa(ij, AJ)) * f
            c3 = (T(ij, TJ, W3) * Aa(ij, AIJ) + T(ij, TJ, W3) * Aa(ij, AJ) + T(im1j, TI, W3) * Aa(ij, AJ)
                  - T(im1j, TI, W3) * Aa(im1j, AI)) * f
            c4 = (T(im1j, TI, W1) * Aa(ij, AJ) - T(im1j, TI, W1) * Aa(im1j, AI) - T(im1jm1, TJ, W3) * Aa(im1j, AI)
                  - T(im1jm1, TJ, W3) * Aa(im1jm1, AIJ)) * f
            c5 = (-T(im1jm1, TJ, W1) * Aa(im1j, AI) - T(im1jm1, TJ, W1) * Aa(im1jm1, AIJ)
                  - T(im1jm1, TI, W1) * Aa(im1jm1, AIJ) - T(im1jm1, TI, W1) * Aa(ijm1, AJ)) * f
            c6 = (-T(im1jm1, TI, W2) * Aa(im1jm1, AIJ) - T(im1jm1, TI, W2) * Aa(ijm1, AJ)
                  - T(ijm1, TJ, W1) * Aa(ijm1, AJ) + T(ijm1, TJ, W1) * Aa(ij, AI)) * f
            for n, cn in enumerate((c0, c1, c2, c3, c4, c5, c6)):
                cg[:, d, n, ij] = cn
            # pentagon at (gmin,gmin)
            p = np.array([(self.gmin - 1) * G + self.gmin - 1])
            pm1j, pm1jm1, pjm1 = p - 1, p - G - 1, p - G
            fp = 0.5 * rarea[:, p]
            for l in np.nonzero(self.have_sgp)[0]:
                def t_(c, t, w):
                    return gt[w, t][l, c]

                def a_(c, a):
                    return ga[d, a][l, c]

                cg[l, d, 0, p] = (t_(p, TI, W1) * a_(p, AI) + t_(p, TI, W1) * a_(p, AIJ) + t_(p, TJ, W1) * a_(p, AIJ)
                                  + t_(p, TJ, W1) * a_(p, AJ) + t_(pm1j, TI, W2) * a_(p, AJ)
                                  - t_(pm1j, TI, W2) * a_(pm1j, AI) - t_(pm1jm1, TJ, W2) * a_(pm1j, AI)
                                  - t_(pm1jm1, TJ, W2) * a_(pm1jm1, AIJ) - t_(pjm1, TJ, W3) * a_(pm1jm1, AIJ)
                                  + t_(pjm1, TJ, W3) * a_(p, AI) - 2 * a_(p, AIJ) - 2 * a_(p, AJ)
                                  + 2 * a_(pm1j, AI) + 2 * a_(pm1jm1, AIJ) - 2 * a_(p, AI)) * fp[l]
                cg[l, d, 1, p] = (-t_(pjm1, TJ, W2) * a_(pm1jm1, AIJ) + t_(pjm1, TJ, W2) * a_(p, AI)
                                  + t_(p, TI, W2) * a_(p, AI) + t_(p, TI, W2) * a_(p, AIJ)) * fp[l]
                cg[l, d, 5, p] = (-t_(pm1jm1, TJ, W1) * a_(pm1j, AI) - t_(pm1jm1, TJ, W1) * a_(pm1jm1, AIJ)) * fp[l]
                cg[l, d, 6, p] = (-t_(pjm1, TJ, W1) * a_(pm1jm1, AIJ) + t_(pjm1, TJ, W1) * a_(p, AI)) * fp[l]
        # poles (mod_oprt.f90:705-731)
        gt_pl, ga_pl, gp_pl = A["GMTR_t_pl"], A["GMTR_a_pl"], A["GMTR_p_pl"]
        cg_pl = np.zeros((2, 3, 6))
        for l in range(2):
            f = 0.5 * gp_pl[1, l, 0]
            for d in range(3):
                s = 0.0
                for v in range(2, 7):
                    vp = 2 if v == 6 else v + 1
                    s += 2.0 * (gt_pl[2, l, v - 1] - 1.0) * ga_pl[d, l, vp - 1]
                cg_pl[l, d, 0] = s * f
                for v in range(2, 7):
                    vp = 2 if v == 6 else v + 1
                    vm = 6 if v == 2 else v - 1
                    cg_pl[l, d, v - 1] = (gt_pl[4, l, vm - 1] * ga_pl[d, l, vm - 1] + gt_pl[4, l, vm - 1] * ga_pl[d, l, v - 1]
                                          + gt_pl[3, l, v - 1] * ga_pl[d, l, v - 1] + gt_pl[3, l, v - 1] * ga_pl[d, l, vp - 1]) * f
        A["coef_grad"] = np.ascontiguousarray(cg)
        A["coef_grad_pl"] = np.ascontiguousarray(cg_pl)

    # ------------------------------------------------------------------
    def geometry(self):
        """The metrics horizontal_flux reads, as passed to ica_set_geometry."""
        A = self.arrays
        return {k: A[k] for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                                  "GMTR_a", "GMTR_a_pl")}

    def interior_mask(self):
        """(lall, gall) bool: cells with gmin <= i,j <= gmax."""
        m = np.zeros((self.lall, self.gall_1d, self.gall_1d), bool)
        m[:, self.gmin - 1:self.gmax, self.gmin - 1:self.gmax] = True
        return m.reshape(self.lall, self.gall)


def default_dt(glevel, dt5=1200.0):
    """dt = 1200 s at glevel 5, scaled by 2^(5-glevel) (Courant number kept near 0.85)."""
    return dt5 * 2.0 ** (5 - glevel)
