"""Seeded inputs for the kernel parity tests, built from the synthetic grid and
fields and passed through the oracle where a kernel's inputs are another
kernel's outputs (flux -> Courant numbers -> remap -> limiter)."""
import functools

import numpy as np

from icoatmosbenchmark_v1_b200 import fields as F
from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
from oracle import oracle as O


@functools.lru_cache(maxsize=8)
def case(glevel=5, rlevel=0, kall=12, ntr=1, kind="mixed"):
    g = Grid(glevel, rlevel, kall)
    f = {k: v.numpy() for k, v in F.make_fields(g).items()}
    st = {k: v.numpy() for k, v in F.make_state(g, ntr, kind).items()}
    d = O.make_dims(glevel, rlevel, kall)
    topo = O.Topo(glevel, rlevel, 1)
    dt = default_dt(glevel)
    geo = g.geometry()
    flx, flx_pl, xc, xc_pl = O.horizontal_flux(d, g.have_sgp, f["rhog"], f["rhog_pl"], f["rhogvx"], f["rhogvx_pl"],
                                               f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], dt, geo)
    ch, ch_pl, cm, cm_pl = O.courant(d, flx, flx_pl, f["rhog"], f["rhog_pl"])
    q = np.ascontiguousarray(st["rhogq"][0] / st["rhog"])
    q_pl = np.ascontiguousarray(st["rhogq_pl"][0] / st["rhog_pl"])
    gr, gr_pl = O.gradient(d, g.have_sgp, q, q_pl, g.arrays)
    topo.data_transfer([gr], [gr_pl])
    qa, qa_pl = O.remap(d, q, q_pl, gr, gr_pl, cm, cm_pl, xc, xc_pl, g.arrays)
    rng = np.random.default_rng(7)
    dd = rng.standard_normal(q.shape) * 1e-3
    dd_pl = rng.standard_normal(q_pl.shape) * 1e-3
    return dict(grid=g, fields=f, state=st, dims=d, topo=topo, dt=dt, geo=geo, flx=flx, flx_pl=flx_pl, xc=xc,
                xc_pl=xc_pl, ch=ch, ch_pl=ch_pl, cm=cm, cm_pl=cm_pl, q=q, q_pl=q_pl, qa=qa, qa_pl=qa_pl,
                d=dd, d_pl=dd_pl)


def vertical_inputs(c):
    """q_h, ck as the composed step builds them (oracle_step.c: vertical sub-step)."""
    g, f = c["grid"], c["fields"]
    K = g.kall
    q, q_pl = c["q"], c["q_pl"]
    af, bf, rdgz = g.arrays["afact"], g.arrays["bfact"], g.arrays["rdgz"]
    rho, rho_pl, w, w_pl = f["rhog"], f["rhog_pl"], f["rhogw"], f["rhogw_pl"]
    dt = c["dt"]

    def build(q, rho, w):
        ck = np.zeros((2,) + q.shape)
        qh = np.zeros_like(q)
        for k in range(1, K - 1):  # 0-based levels kmin-1..kmax-1
            ck[0, :, k] = -w[:, k] * dt * rdgz[k] / rho[:, k]
            ck[1, :, k] = w[:, k + 1] * dt * rdgz[k] / rho[:, k]
        ck[0, :, K - 1] = -w[:, K - 1] * dt * rdgz[K - 1] / rho[:, K - 1]
        for k in range(1, K):
            qh[:, k] = af[k] * q[:, k] + bf[k] * q[:, k - 1]
        return np.ascontiguousarray(qh), np.ascontiguousarray(ck)

    qh, ck = build(q, rho, w)
    qh_pl, ck_pl = build(q_pl, rho_pl, w_pl)
    return qh, qh_pl, ck, ck_pl


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b|."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / den)


def qout_mask(ch, ch_pl, thr=1e-2, tiny=1e-12):
    """Cells whose Thuburn outflow bounds Qout can be compared between precisions
    (regions (lall,K,gall); poles (2,K)).  Two kinds are left out:
    * outflow Courant sum Cout = sum_m max(ch_m, 0) in (0, thr): the bounds are
      (q - qnmax) / Cout + ..., and the FP32 and FP64 builds of the reference switch
      to the zero-outflow form below their own EPS (1.2e-7 vs 2.2e-16), so in between
      they return values that differ by orders of magnitude;
    * a face with 0 < |ch| < tiny: the upwind mask of a face comes from its owner's
      Courant number and the inflow sum from this cell's, and at rounding level the
      two can disagree, which adds ch * (+-HUGE) to the bound (about 1e290 in FP64,
      1e20 in FP32).  Both are properties of the reference algorithm, not of a build."""
    cout = np.maximum(ch, 0).sum(axis=0)
    odd = ((np.abs(ch) > 0) & (np.abs(ch) < tiny)).any(axis=0)
    chp = ch_pl[..., 1:]
    cout_pl = np.maximum(chp, 0).sum(axis=-1)
    odd_pl = ((np.abs(chp) > 0) & (np.abs(chp) < tiny)).any(axis=-1)
    return ((cout == 0) | (cout >= thr)) & ~odd, ((cout_pl == 0) | (cout_pl >= thr)) & ~odd_pl


def interior(a, grid):
    """Values of a (..., lall, K, gall) at interior cells: shape (..., K, n_interior)."""
    m = grid.interior_mask()
    return np.moveaxis(np.asarray(a), -3, -2)[..., m]
