"""Python binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests/,
__graft_entry__.smoke() and the CPU legs of bench.py import it; the product
package icoatmosbenchmark_v1_b200 never does.

Arrays are numpy float64, C-contiguous, in the reference's layout written in
C order: var(gall,kall,lall,m) is shape (m, lall, kall, gall); pole arrays
var_pl(6,kall,2,m) are shape (m, 2, kall, 6).  See icoadv_oracle.h for what
each function restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


class Dims(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("glevel", "rlevel", "kall", "kmin", "kmax", "lall", "have_pl",
                                       "gall_1d", "gall", "gmin", "gmax", "gall_pl", "lall_pl")]


def build():
    srcs = list(HERE.glob("*.c")) + list(HERE.glob("*.h")) + [HERE / "Makefile"]
    if not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB_PATH))
        _lib.orc_topo_create.restype = C.c_void_p
        _lib.orc_topo_create.argtypes = [C.c_int, C.c_int, C.c_int]
        for f in ("orc_topo_destroy",):
            getattr(_lib, f).argtypes = [C.c_void_p]
        for f in ("orc_topo_lall", "orc_topo_rgn_nmax"):
            getattr(_lib, f).argtypes = [C.c_void_p]
        for f in ("orc_topo_have_sgp", "orc_topo_rgnid", "orc_topo_rellist_nmax"):
            getattr(_lib, f).argtypes = [C.c_void_p, C.c_int] + ([C.c_int] if f != "orc_topo_rellist_nmax" else [])
        _lib.orc_topo_rgn4pl.argtypes = [C.c_void_p, C.c_int]
        _lib.orc_topo_edge_tab.argtypes = [C.c_void_p, IP]
        _lib.orc_topo_vert_num.argtypes = [C.c_void_p, IP]
        _lib.orc_comm_data_transfer.argtypes = [C.c_void_p, C.POINTER(DP), C.POINTER(DP), C.c_int, C.c_int]
        _lib.orc_comm_var.argtypes = [C.c_void_p, C.POINTER(DP), C.POINTER(DP), C.c_int, C.c_int]
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(DP)


def make_dims(glevel, rlevel, kall, kmin=None, kmax=None, lall=None, have_pl=1):
    d = Dims(glevel=glevel, rlevel=rlevel, kall=kall,
             kmin=2 if kmin is None else kmin, kmax=(kall - 1) if kmax is None else kmax,
             lall=(10 * 4 ** rlevel) if lall is None else lall, have_pl=have_pl)
    lib().orc_dims_fill(C.byref(d))
    return d


class Topo:
    """mod_adm + mod_comm state of `nprocs` emulated MPI ranks."""

    def __init__(self, glevel, rlevel, nprocs=1):
        self.h = lib().orc_topo_create(glevel, rlevel, nprocs)
        if not self.h:
            raise ValueError("invalid number of processes")
        self.glevel, self.rlevel, self.nprocs = glevel, rlevel, nprocs
        self.lall = lib().orc_topo_lall(self.h)
        self.rgn_nmax = lib().orc_topo_rgn_nmax(self.h)
        self.gall_1d = 2 ** (glevel - rlevel) + 2
        self.gall = self.gall_1d ** 2

    def __del__(self):
        try:
            if getattr(self, "h", None) and _lib is not None:
                _lib.orc_topo_destroy(self.h)
        except Exception:  # interpreter shutdown
            pass
        self.h = None

    def have_sgp(self, rank=1):
        return np.array([lib().orc_topo_have_sgp(self.h, rank, l) for l in range(1, self.lall + 1)], np.int32)

    def rgnid(self, rank, l):
        return lib().orc_topo_rgnid(self.h, rank, l)

    def rgn4pl(self, pole):
        return lib().orc_topo_rgn4pl(self.h, pole)

    def rellist_nmax(self, rank):
        return lib().orc_topo_rellist_nmax(self.h, rank)

    def edge_tab(self):
        out = np.zeros((self.rgn_nmax, 4, 2), np.int32)
        lib().orc_topo_edge_tab(self.h, out.ctypes.data_as(IP))
        return out

    def vert_num(self):
        out = np.zeros((self.rgn_nmax, 4), np.int32)
        lib().orc_topo_vert_num(self.h, out.ctypes.data_as(IP))
        return out

    def _call(self, fn, var, var_pl):
        kmax, vmax = var[0].shape[2], var[0].shape[0]
        va = (DP * self.nprocs)(*[_p(v) for v in var])
        pa = (DP * self.nprocs)(*[_p(v) for v in var_pl])
        fn(self.h, va, pa, kmax, vmax)

    def data_transfer(self, var, var_pl):
        """COMM_data_transfer over all ranks, in place.  var[rank] shape (vmax, lall, kmax, gall)."""
        self._call(lib().orc_comm_data_transfer, var, var_pl)

    def comm_var(self, var, var_pl):
        self._call(lib().orc_comm_var, var, var_pl)


def _sgp(have_sgp):
    a = np.ascontiguousarray(have_sgp, dtype=np.int32)
    return a, a.ctypes.data_as(IP)


def horizontal_flux(d, have_sgp, rho, rho_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, dt, geo):
    L, K, G = d.lall, d.kall, d.gall
    flx = np.zeros((6, L, K, G)); flx_pl = np.zeros((2, K, 6))
    xc = np.zeros((3, 3, L, K, G)); xc_pl = np.zeros((3, 2, K, 6))
    s, sp = _sgp(have_sgp)
    lib().orc_horizontal_flux(C.byref(d), sp, _p(flx), _p(flx_pl), _p(xc), _p(xc_pl), _p(rho), _p(rho_pl),
                              _p(vx), _p(vx_pl), _p(vy), _p(vy_pl), _p(vz), _p(vz_pl), C.c_double(dt),
                              _p(geo["GRD_xr"]), _p(geo["GRD_xr_pl"]), _p(geo["GMTR_p"]), _p(geo["GMTR_p_pl"]),
                              _p(geo["GMTR_t"]), _p(geo["GMTR_t_pl"]), _p(geo["GMTR_a"]), _p(geo["GMTR_a_pl"]))
    return flx, flx_pl, xc, xc_pl


def horizontal_limiter(d, have_sgp, q_a, q_a_pl, q, q_pl, dd, d_pl, ch, ch_pl, cmask, cmask_pl,
                       Qout_post=None, Qout_post_pl=None, topo=None):
    """Returns (q_a, q_a_pl, Qout_prev, Qout_prev_pl); q_a inputs are not modified."""
    q_a = q_a.copy(); q_a_pl = q_a_pl.copy()
    L, K, G = d.lall, d.kall, d.gall
    qo = np.zeros((2, L, K, G)); qo_pl = np.zeros((2, 2, K, 6))
    s, sp = _sgp(have_sgp)
    if Qout_post is None and topo is None:
        raise ValueError("need Qout_post or a single-rank topology")
    lib().orc_horizontal_limiter_thuburn(C.byref(d), sp, _p(q_a), _p(q_a_pl), _p(q), _p(q_pl), _p(dd), _p(d_pl),
                                         _p(ch), _p(ch_pl), _p(cmask), _p(cmask_pl), _p(qo), _p(qo_pl),
                                         _p(Qout_post), _p(Qout_post_pl),
                                         C.c_void_p(topo.h) if topo is not None else None)
    return q_a, q_a_pl, qo, qo_pl


def vertical_limiter(d, q_h, q_h_pl, q, q_pl, dd, d_pl, ck, ck_pl):
    q_h = q_h.copy(); q_h_pl = q_h_pl.copy()
    lib().orc_vertical_limiter_thuburn(C.byref(d), _p(q_h), _p(q_h_pl), _p(q), _p(q_pl), _p(dd), _p(d_pl),
                                       _p(ck), _p(ck_pl))
    return q_h, q_h_pl


def gradient(d, have_sgp, q, q_pl, geo):
    L, K, G = d.lall, d.kall, d.gall
    gr = np.zeros((3, L, K, G)); gr_pl = np.zeros((3, 2, K, 6))
    s, sp = _sgp(have_sgp)
    lib().orc_gradient(C.byref(d), sp, _p(gr), _p(gr_pl), _p(q), _p(q_pl), _p(geo["coef_grad"]),
                       _p(geo["coef_grad_pl"]))
    return gr, gr_pl


def courant(d, flx, flx_pl, rho, rho_pl):
    ch = np.zeros_like(flx); ch_pl = np.zeros_like(flx_pl)
    cm = np.zeros_like(flx); cm_pl = np.zeros_like(flx_pl)
    lib().orc_courant(C.byref(d), _p(ch), _p(ch_pl), _p(cm), _p(cm_pl), _p(flx), _p(flx_pl), _p(rho), _p(rho_pl))
    return ch, ch_pl, cm, cm_pl


def remap(d, q, q_pl, gr, gr_pl, cm, cm_pl, xc, xc_pl, geo):
    L, K, G = d.lall, d.kall, d.gall
    qa = np.zeros((6, L, K, G)); qa_pl = np.zeros((2, K, 6))
    lib().orc_remap(C.byref(d), _p(qa), _p(qa_pl), _p(q), _p(q_pl), _p(gr), _p(gr_pl), _p(cm), _p(cm_pl),
                    _p(xc), _p(xc_pl), _p(geo["GRD_x"]), _p(geo["GRD_x_pl"]))
    return qa, qa_pl


def step_adjoint(d, have_sgp, topo, dt, state, fields, geo, adj_state, adj_wind):
    """Adjoint of one step at input `state`: adj_state (rhog, rhog_pl, rhogq, rhogq_pl) holds the
    adjoint of the step's output and is overwritten with the adjoint of its input; adj_wind
    (rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz, rhogvz_pl) is accumulated."""
    s, sp = _sgp(have_sgp)
    ntr = state["rhogq"].shape[0]
    lib().orc_step_adjoint(C.byref(d), sp, C.c_void_p(topo.h), ntr, C.c_double(dt),
                           _p(state["rhog"]), _p(state["rhog_pl"]), _p(state["rhogq"]), _p(state["rhogq_pl"]),
                           _p(fields["rhogvx"]), _p(fields["rhogvx_pl"]), _p(fields["rhogvy"]),
                           _p(fields["rhogvy_pl"]), _p(fields["rhogvz"]), _p(fields["rhogvz_pl"]),
                           _p(fields["rhogw"]), _p(fields["rhogw_pl"]),
                           _p(geo["rdgz"]), _p(geo["afact"]), _p(geo["bfact"]),
                           _p(geo["GRD_x"]), _p(geo["GRD_x_pl"]), _p(geo["GRD_xr"]), _p(geo["GRD_xr_pl"]),
                           _p(geo["GMTR_p"]), _p(geo["GMTR_p_pl"]), _p(geo["GMTR_t"]), _p(geo["GMTR_t_pl"]),
                           _p(geo["GMTR_a"]), _p(geo["GMTR_a_pl"]), _p(geo["coef_grad"]), _p(geo["coef_grad_pl"]),
                           _p(adj_state["rhog"]), _p(adj_state["rhog_pl"]), _p(adj_state["rhogq"]),
                           _p(adj_state["rhogq_pl"]), _p(adj_wind["rhogvx"]), _p(adj_wind["rhogvx_pl"]),
                           _p(adj_wind["rhogvy"]), _p(adj_wind["rhogvy_pl"]), _p(adj_wind["rhogvz"]),
                           _p(adj_wind["rhogvz_pl"]))


def step(d, have_sgp, topo, dt, state, fields, geo, nthreads=None):
    """One composed tracer step in place on state = dict(rhog, rhog_pl, rhogq, rhogq_pl)."""
    s, sp = _sgp(have_sgp)
    ntr = state["rhogq"].shape[0]
    nthreads = nthreads or os.cpu_count() or 1
    lib().orc_step(C.byref(d), sp, C.c_void_p(topo.h), ntr, C.c_double(dt),
                   _p(state["rhog"]), _p(state["rhog_pl"]), _p(state["rhogq"]), _p(state["rhogq_pl"]),
                   _p(fields["rhogvx"]), _p(fields["rhogvx_pl"]), _p(fields["rhogvy"]), _p(fields["rhogvy_pl"]),
                   _p(fields["rhogvz"]), _p(fields["rhogvz_pl"]), _p(fields["rhogw"]), _p(fields["rhogw_pl"]),
                   _p(geo["rdgz"]), _p(geo["afact"]), _p(geo["bfact"]),
                   _p(geo["GRD_x"]), _p(geo["GRD_x_pl"]), _p(geo["GRD_xr"]), _p(geo["GRD_xr_pl"]),
                   _p(geo["GMTR_p"]), _p(geo["GMTR_p_pl"]), _p(geo["GMTR_t"]), _p(geo["GMTR_t_pl"]),
                   _p(geo["GMTR_a"]), _p(geo["GMTR_a_pl"]), _p(geo["coef_grad"]), _p(geo["coef_grad_pl"]),
                   int(nthreads))


class GridTables:
    """Region topology and composed halo plan from this oracle's restatement of the
    reference's mod_adm / mod_comm (one emulated rank), in the form the synthetic grid
    builder takes (icoatmosbenchmark_v1_b200.grid.Grid(tables=...)), so that a grid can be
    built without the library under test.  The plan is read off COMM_data_transfer itself:
    every point starts holding its own flat index, and after the transfer a point that
    holds another index is a destination whose source is that index."""

    def topology_info(self, glevel, rlevel):
        t = Topo(glevel, rlevel, 1)
        return t.have_sgp(1), np.array([t.rgn4pl(1), t.rgn4pl(2)], np.int32), None

    def comm_plan(self, glevel, rlevel, pole_fill=False):
        t = Topo(glevel, rlevel, 1)
        L, G = t.lall, t.gall
        var = np.arange(L * G, dtype=np.float64).reshape(1, L, 1, G)
        var_pl = (L * G + np.arange(12, dtype=np.float64)).reshape(1, 2, 1, 6)
        (t.comm_var if pole_fill else t.data_transfer)([var], [var_pl])
        flat = np.concatenate([var.reshape(-1), var_pl.reshape(-1)]).astype(np.int64)
        dst = np.nonzero(flat != np.arange(flat.size))[0]
        return dst.astype(np.int32), flat[dst].astype(np.int32)
