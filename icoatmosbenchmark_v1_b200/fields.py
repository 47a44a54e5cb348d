"""Synthetic fields of the benchmark configurations (seeded), built with torch
so the large configurations can be generated directly in device memory.

Per configuration (rl 0, R = 6.371e6 m):
  rho   = 1.2 exp(-z/8000) kg/m^3 at full levels
  v     = solid-body rotation, 40 m/s at the rotation equator (axis tilted 45 deg
          towards +x so the flow crosses both poles), plus Gaussian noise of
          2 m/s std projected on the sphere's tangent plane and smoothed by 3
          passes of neighbour averaging
  rhogv = rho v; the noise is a column-mass-neutral baroclinic mode and rhogw comes
          from the discrete continuity equation, so rho stays steady (see make_fields)
  tracers in [0,1]: "bell" = cosine bell of radius R/3 plus a slotted cylinder
          (per tracer the two centres rotate in longitude), "smooth" = random
          field of real spherical harmonics of degree <= 16 (seeded
          coefficients) scaled about 0.5 and clipped to [0,1];
          each with a vertical profile that steps at 12 km so the vertical
          limiter is active.
Seeds: numpy PCG64(20261203) for the noise, tracer i uses seed 20261203 + 1 + i.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .grid import Grid

SEED = 20261203


def _flat(var, var_pl):
    """(m, L, K, G), (m, 2, K, 6) -> (m, K, L*G + 12)."""
    m, L, K, G = var.shape
    return torch.cat([var.permute(0, 2, 1, 3).reshape(m, K, L * G), var_pl.permute(0, 2, 1, 3).reshape(m, K, 12)], 2)


def _unflat(flat, L, G):
    m, K, _ = flat.shape
    var = flat[:, :, :L * G].reshape(m, K, L, G).permute(0, 2, 1, 3).contiguous()
    var_pl = flat[:, :, L * G:].reshape(m, K, 2, 6).permute(0, 2, 1, 3).contiguous()
    return var, var_pl


def halo_fill(grid: Grid, var, var_pl):
    """Single-process halo/pole fill with the composed COMM plan (host-side preparation of inputs)."""
    dst, src = grid.plan
    f = _flat(var, var_pl)
    d = torch.as_tensor(dst, device=f.device, dtype=torch.long)
    s = torch.as_tensor(src, device=f.device, dtype=torch.long)
    f[:, :, d] = f[:, :, s]
    return _unflat(f, grid.lall, grid.gall)


def _positions(grid: Grid, device):
    x = torch.as_tensor(grid.arrays["GRD_x"], device=device) / grid.R  # (3, L, gall)
    xp = torch.as_tensor(grid.arrays["GRD_x_pl"], device=device) / grid.R  # (3, 2, 6)
    return x, xp


def _smooth_columns(grid: Grid, v, vp, passes=3):
    """Neighbour averaging (self + 6 hexagon neighbours) on interior cells; poles average their ring."""
    L, G = grid.lall, grid.gall_1d
    g0, g1 = grid.gmin - 1, grid.gmax - 1
    for _ in range(passes):
        a = v.reshape(v.shape[0], L, v.shape[2], G, G)
        c = a[..., g0:g1 + 1, g0:g1 + 1]
        s = (c + a[..., g0:g1 + 1, g0 + 1:g1 + 2] + a[..., g0 + 1:g1 + 2, g0 + 1:g1 + 2] + a[..., g0 + 1:g1 + 2, g0:g1 + 1]
             + a[..., g0:g1 + 1, g0 - 1:g1] + a[..., g0 - 1:g1, g0 - 1:g1] + a[..., g0 - 1:g1, g0:g1 + 1]) / 7.0
        a = a.clone()
        a[..., g0:g1 + 1, g0:g1 + 1] = s
        vp = vp.clone()
        vp[..., 0] = vp.sum(-1) / 6.0
        v, vp = halo_fill(grid, a.reshape(v.shape), vp)
    return v, vp


def mass_flux_divergence(grid: Grid, rho, rhov, rho_pl, rhov_pl):
    """Horizontal mass-flux divergence sum_m flx_h(m) / dt per cell and level (FP64), with the
    face fluxes of horizontal_flux (triangle interpolation, singular point, pentagon face);
    interior cells and the pole centres.  rho (L,K,gall), rhov (3,L,K,gall); poles (2,K,6)."""
    A = grid.arrays
    L, K, G = grid.lall, rho.shape[1], grid.gall_1d
    dev = rho.device
    gt = torch.as_tensor(A["GMTR_t"], device=dev).view(5, 2, L, 1, G, G)
    ga = torch.as_tensor(A["GMTR_a"], device=dev).view(12, 3, L, 1, G, G)
    ra = torch.as_tensor(A["GMTR_p"][1], device=dev).view(L, 1, G, G)
    f = torch.stack([rho, rhov[0], rhov[1], rhov[2]]).view(4, L, K, G, G)  # [..., j, i]
    s0, s1 = slice(0, G - 1), slice(1, G)
    TI = f[..., s0, s0] * gt[2, 0][..., s0, s0] + f[..., s0, s1] * gt[3, 0][..., s0, s0]
    TI = TI + f[..., s1, s1] * gt[4, 0][..., s0, s0]
    TJ = f[..., s0, s0] * gt[2, 1][..., s0, s0]
    TJ = TJ + f[..., s1, s1] * gt[3, 1][..., s0, s0] + f[..., s1, s0] * gt[4, 1][..., s0, s0]
    sg = torch.as_tensor(grid.have_sgp, device=dev).bool()
    TI[:, sg, :, 0, 0] = TJ[:, sg, :, 0, 1]  # rhot_TI(gmin-1,gmin-1) = rhot_TJ(gmin,gmin-1)

    def face(v, a, jj, ii):  # 0.5 (v . HN) of face a at owners [jj, ii]
        return 0.5 * (v[1] * ga[0, a][..., jj, ii] + v[2] * ga[1, a][..., jj, ii] + v[3] * ga[2, a][..., jj, ii])

    n = G - 2  # interior cells 0-based 1..G-2
    ci, cm = slice(1, G - 1), slice(0, G - 2)
    fai = face(TJ[..., cm, ci] + TI[..., ci, ci], 0, ci, ci)           # AI of (i,j)
    faim = face(TJ[..., cm, cm] + TI[..., ci, cm], 0, ci, cm)          # AI of (i-1,j)
    faij = face(TI[..., ci, ci] + TJ[..., ci, ci], 1, ci, ci)          # AIJ of (i,j)
    faijm = face(TI[..., cm, cm] + TJ[..., cm, cm], 1, cm, cm)         # AIJ of (i-1,j-1)
    faj = face(TJ[..., ci, ci] + TI[..., ci, cm], 2, ci, ci)           # AJ of (i,j)
    fajm = face(TJ[..., cm, ci] + TI[..., cm, cm], 2, cm, ci)          # AJ of (i,j-1)
    fajm[sg, :, 0, 0] = 0.0  # flx_h(gmin,gmin,6) = 0
    div = ra[..., ci, ci] * (fai + faij + faj - faim - faijm - fajm)
    out = torch.zeros(L, K, G, G, dtype=rho.dtype, device=dev)
    out[:, :, 1:G - 1, 1:G - 1] = div
    # poles
    gtp = torch.as_tensor(A["GMTR_t_pl"], device=dev)
    gap = torch.as_tensor(A["GMTR_a_pl"], device=dev)
    rap = torch.as_tensor(A["GMTR_p_pl"][1][:, 0], device=dev)
    fp = torch.stack([rho_pl, rhov_pl[0], rhov_pl[1], rhov_pl[2]])  # (4, 2, K, 6)
    out_pl = torch.zeros_like(rho_pl)
    for p in range(2):
        T = {}
        for v in range(2, 7):
            vp = 2 if v == 6 else v + 1
            T[v] = fp[:, p, :, 0] * gtp[2, p, v - 1] + fp[:, p, :, v - 1] * gtp[3, p, v - 1] + fp[:, p, :, vp - 1] * gtp[4, p, v - 1]
        tot = 0.0
        for v in range(2, 7):
            vm = 6 if v == 2 else v - 1
            vv = T[vm] + T[v]
            tot = tot + 0.5 * (vv[1] * gap[0, p, v - 1] + vv[2] * gap[1, p, v - 1] + vv[3] * gap[2, p, v - 1])
        out_pl[p, :, 0] = rap[p] * tot
    return out.view(L, K, G * G), out_pl


def make_fields(grid: Grid, device="cpu", u0=40.0, noise=2.0, alpha=math.pi / 4, seed=SEED,
                dtype=torch.float64):
    """Shared per-step fields: rho, rhogvx/vy/vz (cell centres), rhogw (faces below each level).

    The horizontal noise is a baroclinic, column-mass-neutral mode: a smoothed random tangent field
    times a vertical profile A(z) with sum_k rho A dz = 0, RMS 2 m/s.  rhogw then follows from the
    discrete continuity equation integrated upward from the ground (rhogw = 0 there and at the top),
    so the density stays steady step after step (the literal per-level random w and divergent
    noise drive rho to zero within a few steps once rho is advanced by the continuity equation)."""
    L, K, gall = grid.lall, grid.kall, grid.gall
    vg = grid.arrays
    z = torch.as_tensor(vg["z"], device=device)
    dz = torch.as_tensor(vg["dz"], device=device)
    rho_k = 1.2 * torch.exp(-z / 8000.0)
    rho = rho_k.view(1, K, 1).expand(L, K, gall).contiguous()
    rho_pl = rho_k.view(1, K, 1).expand(2, K, 6).contiguous()
    x, xp = _positions(grid, device)
    axis = torch.tensor([math.sin(alpha), 0.0, math.cos(alpha)], device=device, dtype=torch.float64)

    def rot(p):  # axis x p, p (3, ...)
        return torch.stack([axis[1] * p[2] - axis[2] * p[1], axis[2] * p[0] - axis[0] * p[2],
                            axis[0] * p[1] - axis[1] * p[0]])

    rng = np.random.Generator(np.random.PCG64(seed))
    nz = torch.as_tensor(rng.standard_normal((3, L, 1, gall)), device=device)
    nzp = torch.as_tensor(rng.standard_normal((3, 2, 1, 6)), device=device)
    xe, xpe = x.unsqueeze(2), xp.unsqueeze(2)  # (3, L, 1, gall)
    nz = nz - (nz * xe).sum(0, keepdim=True) * xe
    nzp = nzp - (nzp * xpe).sum(0, keepdim=True) * xpe
    nz, nzp = halo_fill(grid, nz, nzp)
    nz, nzp = _smooth_columns(grid, nz, nzp)
    sd = torch.cat([nz.reshape(3, -1), nzp.reshape(3, -1)], 1).norm(dim=0).pow(2).mean().sqrt()
    # vertical profile of the noise: one sign change, zero mass-weighted column mean, unit RMS
    phys = torch.zeros(K, dtype=torch.bool, device=device)
    phys[grid.kmin - 1:grid.kmax] = True
    prof = torch.cos(math.pi * z / 40.0e3)
    c = (rho_k * prof * dz)[phys].sum() / (rho_k * dz)[phys].sum()
    prof = torch.where(phys, prof - c, torch.zeros_like(prof))
    prof = prof / prof[phys].pow(2).mean().sqrt()
    v = u0 * rot(xe) + noise * (nz / sd) * prof.view(1, 1, K, 1)
    vp = u0 * rot(xpe) + noise * (nzp / sd) * prof.view(1, 1, K, 1)
    rhogv = v * rho.unsqueeze(0)
    rhogv_pl = vp * rho_pl.unsqueeze(0)
    rhogv, rhogv_pl = halo_fill(grid, rhogv, rhogv_pl)
    # vertical mass flux from continuity: rhogw(k+1) = rhogw(k) - hdiv(k) dz(k), ground and top = 0
    hdiv, hdiv_pl = mass_flux_divergence(grid, rho, rhogv, rho_pl, rhogv_pl)
    rhogw = torch.zeros(L, K, gall, dtype=torch.float64, device=device)
    rhogw_pl = torch.zeros(2, K, 6, dtype=torch.float64, device=device)
    for k in range(grid.kmin - 1, grid.kmax):  # faces kmin+1 .. kmax+1 (0-based k+1)
        rhogw[:, k + 1] = rhogw[:, k] - hdiv[:, k] * dz[k]
        rhogw_pl[:, k + 1] = rhogw_pl[:, k] - hdiv_pl[:, k] * dz[k]
    # the column's net divergence (residual flux through the top) is spread over the column by
    # mass, so the top flux is zero and rho changes by the same small fraction at every level
    top = grid.kmax  # 0-based index of the top face kmax+1
    cum = torch.zeros(K, dtype=torch.float64, device=device)
    cum[grid.kmin - 1:top + 1] = torch.cat([torch.zeros(1, dtype=torch.float64, device=device),
                                            torch.cumsum((rho_k * dz)[grid.kmin - 1:top], 0)])
    cum = cum / cum[top]
    rhogw = rhogw - rhogw[:, top:top + 1] * cum.view(1, K, 1)
    rhogw_pl = rhogw_pl - rhogw_pl[:, top:top + 1] * cum.view(1, K, 1)
    rhogw[:, top] = 0.0
    rhogw_pl[:, top] = 0.0
    rhogw, rhogw_pl = halo_fill(grid, rhogw.unsqueeze(0), rhogw_pl.unsqueeze(0))
    out = dict(rhog=rho, rhog_pl=rho_pl, rhogvx=rhogv[0], rhogvx_pl=rhogv_pl[0], rhogvy=rhogv[1],
               rhogvy_pl=rhogv_pl[1], rhogvz=rhogv[2], rhogvz_pl=rhogv_pl[2], rhogw=rhogw[0], rhogw_pl=rhogw_pl[0])
    return {k: t.to(dtype).contiguous() for k, t in out.items()}


def _bell_cylinder(x, lon0, lat0, R_frac=1.0 / 3.0):
    """Cosine bell (radius R/3) at (lon0,lat0) plus a slotted cylinder 120 deg east of it, in [0,1]."""
    def centre(lon, lat):
        return torch.tensor([math.cos(lat) * math.cos(lon), math.cos(lat) * math.sin(lon), math.sin(lat)],
                            dtype=x.dtype, device=x.device).view(3, *([1] * (x.dim() - 1)))

    r = R_frac  # angular radius (radians) of R/3 on the sphere
    d1 = torch.arccos(torch.clamp((x * centre(lon0, lat0)).sum(0), -1, 1))
    bell = torch.where(d1 < r, 0.5 * (1 + torch.cos(math.pi * d1 / r)), torch.zeros_like(d1))
    c2 = centre(lon0 + 2 * math.pi / 3, lat0)
    d2 = torch.arccos(torch.clamp((x * c2).sum(0), -1, 1))
    # slot: remove a narrow band through the centre along the local meridian
    lon = torch.atan2(x[1], x[0])
    dlon = torch.remainder(lon - (lon0 + 2 * math.pi / 3) + math.pi, 2 * math.pi) - math.pi
    slot = (dlon.abs() < r / 6) & (torch.asin(torch.clamp(x[2], -1, 1)) - lat0 < r * 5 / 6)
    cyl = torch.where((d2 < r) & ~slot, torch.ones_like(d2), torch.zeros_like(d2))
    return torch.clamp(bell + cyl, 0.0, 1.0)


def spherical_harmonic_field(x, seed, lmax=16):
    """Random band-limited field on the unit sphere: sum over degrees l <= lmax and orders
    |m| <= l of a_lm Y_lm(x), real orthonormal spherical harmonics, with seeded coefficients
    a_lm ~ N(0, 1) / (1 + l) (a red spectrum, so the field is smooth at the grid scale).
    x: unit vectors (3, ...).  The associated Legendre functions come from the standard
    fully normalised three-term recurrences in l (stable to l of a few hundred)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    ct = torch.clamp(x[2], -1.0, 1.0)
    st = torch.sqrt(torch.clamp(1.0 - ct * ct, min=0.0))
    phi = torch.atan2(x[1], x[0])
    f = torch.zeros_like(ct)
    pmm = torch.full_like(ct, 1.0 / math.sqrt(4.0 * math.pi))  # P_0^0
    for m in range(lmax + 1):
        if m > 0:
            pmm = -math.sqrt((2.0 * m + 1.0) / (2.0 * m)) * st * pmm
        p_lm2, p_lm1 = None, pmm  # P_{l-2}^m, P_{l-1}^m with l-1 = m
        cm, sm = (torch.cos(m * phi), torch.sin(m * phi)) if m > 0 else (None, None)
        for l in range(m, lmax + 1):
            if l == m:
                p = pmm
            elif l == m + 1:
                p = math.sqrt(2.0 * m + 3.0) * ct * pmm
            else:
                a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
                b = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
                p = a * (ct * p_lm1 - b * p_lm2)
            if l > m:
                p_lm2, p_lm1 = p_lm1, p
            amp = 1.0 / (1.0 + l)
            if m == 0:
                f = f + amp * float(torch.randn(1, generator=g, dtype=torch.float64)) * p
            else:
                c1, c2 = torch.randn(2, generator=g, dtype=torch.float64).tolist()
                f = f + amp * math.sqrt(2.0) * p * (c1 * cm + c2 * sm)
    return f


def _smooth_random(x, seed, lmax=16):
    """Seeded spherical-harmonic field of degree <= lmax, scaled about 0.5 and clipped to [0, 1]."""
    f = spherical_harmonic_field(x, seed, lmax)
    f = 0.5 + 0.5 * f / (f.abs().max() + 1e-30) * 1.2
    return torch.clamp(f, 0.0, 1.0)


def tracer_mixing_ratio(grid: Grid, ntr, kind="bell", device="cpu", seed=SEED):
    """q (ntr, L, K, gall) and q_pl (ntr, 2, K, 6); kind: 'bell', 'smooth' or 'mixed' (half each)."""
    x, xp = _positions(grid, device)
    z = torch.as_tensor(grid.arrays["z"], device=device)
    qs, qps = [], []
    for t in range(ntr):
        k = kind if kind != "mixed" else ("smooth" if t % 2 == 0 else "bell")
        if k == "bell":
            lon0, lat0 = 2 * math.pi * t / max(ntr, 1) + 0.3, 0.4 * math.sin(1.7 * t + 0.5)
            q2, q2p = _bell_cylinder(x, lon0, lat0), _bell_cylinder(xp, lon0, lat0)
        else:
            q2, q2p = _smooth_random(x, seed + 1 + t), _smooth_random(xp, seed + 1 + t)
        prof = torch.where(z < 12.0e3 + 500.0 * t, torch.ones_like(z), 0.35 * torch.ones_like(z))
        qs.append(q2.unsqueeze(1) * prof.view(1, -1, 1))
        qps.append(q2p.unsqueeze(1) * prof.view(1, -1, 1))
    q = torch.stack(qs).contiguous()
    qp = torch.stack(qps).contiguous()
    return halo_fill(grid, q, qp)


def make_state(grid: Grid, ntr, kind="bell", device="cpu", fields=None):
    """Prognostic state: rhog (L,K,gall), rhogq (ntr,L,K,gall) (+ poles), FP64."""
    f = fields if fields is not None else make_fields(grid, device)
    q, qp = tracer_mixing_ratio(grid, ntr, kind, device)
    rhog = f["rhog"].to(torch.float64).clone()
    rhog_pl = f["rhog_pl"].to(torch.float64).clone()
    return dict(rhog=rhog, rhog_pl=rhog_pl, rhogq=(q * rhog.unsqueeze(0)).contiguous(),
                rhogq_pl=(qp * rhog_pl.unsqueeze(0)).contiguous())
