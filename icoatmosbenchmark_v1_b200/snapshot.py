"""Kernel snapshots of IcoAtmosBenchmark_v1 (NICAM kernels) and their point-by-point check.

The reference drivers read one binary snapshot per process, `snapshot.<kernel>.pe<6 digits>`
(`kernels/NICAM/<kernel>/src/main.f90`, via `dumpio.c`): raw 8-byte reals, big-endian, no
record markers, the arrays one after the other in the driver's read order, each in
Fortran (column-major) order.  The expected outputs come first (the driver keeps them as
`check_*` and prints `expected - computed`), then the inputs.  The reference's own
snapshots are for one region of a glevel-7 grid with the poles (`ADM_lall = 1`,
`ADM_gall_1d = 130`, `ADM_kall = 42`, `problem_size.inc`).

This module reads and writes that format (arrays come back in this library's C layout:
Fortran var(ij,k,l,m) is the C array [m][l][k][ij]) and runs a snapshot through the
library as a driver would: a context made by ica_init_regions with the driver's own sizes
(ADM_gall_1d, ADM_kall, ADM_kmin, ADM_kmax, ADM_lall = 1, ADM_have_pl, ADM_have_sgp(1)),
the kernel through its host-pointer entry point on the snapshot's arrays as they are, and
the outputs compared with the expected ones, in the driver's
`+check[name] max=..., min=..., sum=...` form.

    python -m icoatmosbenchmark_v1_b200.snapshot run dyn_horiz_adv_flux snapshot.dyn_horiz_adv_flux.pe000000
"""
from __future__ import annotations

import argparse
import dataclasses
import math
from collections import OrderedDict
from pathlib import Path

import numpy as np

KERNELS = ("dyn_horiz_adv_flux", "dyn_horiz_adv_limiter", "dyn_vert_adv_limiter")

GMTR_P_NMAX, GMTR_T_NMAX, GMTR_A_NMAX, GMTR_A_NMAX_PL = 8, 5, 12, 18  # problem_size.inc:80-100


@dataclasses.dataclass(frozen=True)
class SnapshotDims:
    """Sizes of one process's arrays (ADM_* of problem_size.inc); the defaults are the
    reference's snapshots."""
    gall_1d: int = 130
    kall: int = 42
    lall: int = 1
    gall_pl: int = 6
    lall_pl: int = 2

    @property
    def gall(self):
        return self.gall_1d * self.gall_1d

    @property
    def glevel(self):  # rlevel 0: gall_1d = 2^glevel + 2
        g = int(round(math.log2(self.gall_1d - 2)))
        if 2 ** g + 2 != self.gall_1d:
            raise ValueError(f"gall_1d {self.gall_1d} is not 2^glevel + 2")
        return g


# read order of each driver: name, Fortran extents (symbols G = gall, P = gall_pl, K = kall,
# L = lall, LP = lall_pl, K0 = 1), and whether the driver checks it as an output
def _layout(kernel):
    if kernel == "dyn_horiz_adv_flux":  # dyn_horiz_adv_flux/src/main.f90:145-164
        return [("flx_h", "G K L 6", True), ("flx_h_pl", "P K LP", True),
                ("GRD_xc", "G K L 3 3", True), ("GRD_xc_pl", "P K LP 3", True),
                ("rho", "G K L", False), ("rho_pl", "P K LP", False),
                ("rhovx", "G K L", False), ("rhovx_pl", "P K LP", False),
                ("rhovy", "G K L", False), ("rhovy_pl", "P K LP", False),
                ("rhovz", "G K L", False), ("rhovz_pl", "P K LP", False),
                ("GRD_xr", "G K0 L 3 3", False), ("GRD_xr_pl", "P K0 LP 3", False),
                ("GMTR_p", f"G K0 L {GMTR_P_NMAX}", False), ("GMTR_p_pl", f"P K0 LP {GMTR_P_NMAX}", False),
                ("GMTR_t", f"G K0 L 2 {GMTR_T_NMAX}", False), ("GMTR_t_pl", f"P K0 LP {GMTR_T_NMAX}", False),
                ("GMTR_a", f"G K0 L 3 {GMTR_A_NMAX}", False), ("GMTR_a_pl", f"P K0 LP {GMTR_A_NMAX_PL}", False)]
    if kernel == "dyn_horiz_adv_limiter":  # dyn_horiz_adv_limiter/src/main.f90:132-147
        return [("q_a_prev", "G K L 6", False), ("q_a_prev_pl", "P K LP", False),
                ("q_a", "G K L 6", True), ("q_a_pl", "P K LP", True),
                ("q", "G K L", False), ("q_pl", "P K LP", False),
                ("d", "G K L", False), ("d_pl", "P K LP", False),
                ("ch", "G K L 6", False), ("ch_pl", "P K LP", False),
                ("cmask", "G K L 6", False), ("cmask_pl", "P K LP", False),
                ("Qout_prev", "G K L 2", True), ("Qout_prev_pl", "P K LP 2", True),
                ("Qout_post", "G K L 2", False), ("Qout_post_pl", "P K LP 2", False)]
    if kernel == "dyn_vert_adv_limiter":  # dyn_vert_adv_limiter/src/main.f90:96-105
        return [("q_h_prev", "G K L", False), ("q_h_prev_pl", "P K LP", False),
                ("q_h", "G K L", True), ("q_h_pl", "P K LP", True),
                ("q", "G K L", False), ("q_pl", "P K LP", False),
                ("d", "G K L", False), ("d_pl", "P K LP", False),
                ("ck", "G K L 2", False), ("ck_pl", "P K LP 2", False)]
    raise ValueError(f"unknown kernel {kernel!r}; one of {KERNELS}")


def layout(kernel, dims=SnapshotDims()):
    """[(name, Fortran extents, is_output)] in the driver's read order."""
    sym = {"G": dims.gall, "P": dims.gall_pl, "K": dims.kall, "L": dims.lall, "LP": dims.lall_pl, "K0": 1}
    return [(n, tuple(sym[t] if t in sym else int(t) for t in ext.split()), out) for n, ext, out in _layout(kernel)]


def file_name(kernel, rank=0):
    """dumpio_mk_fname(fname, 'snapshot.<kernel>', 'pe', rank, 6)."""
    return f"snapshot.{kernel}.pe{rank:06d}"


def read_snapshot(kernel, path, dims=SnapshotDims()):
    """The arrays of a snapshot, in read order, as C-layout float64 arrays (Fortran extents
    reversed).  The file must hold exactly the driver's arrays."""
    raw = Path(path).read_bytes()
    lay = layout(kernel, dims)
    need = 8 * sum(int(np.prod(e)) for _, e, _ in lay)
    if len(raw) != need:
        raise ValueError(f"{path}: {len(raw)} bytes, the {kernel} driver reads {need} for {dims}")
    out, pos = OrderedDict(), 0
    for name, ext, _ in lay:
        n = int(np.prod(ext))
        out[name] = np.frombuffer(raw, dtype=">f8", count=n, offset=pos).astype(np.float64).reshape(ext[::-1])
        pos += 8 * n
    return out


def write_snapshot(kernel, path, arrays, dims=SnapshotDims()):
    """Writes arrays (C layout, name -> array) in the driver's read order."""
    parts = []
    for name, ext, _ in layout(kernel, dims):
        a = np.asarray(arrays[name], dtype=np.float64)
        if a.shape != ext[::-1]:
            raise ValueError(f"{name}: shape {a.shape}, the {kernel} driver reads {ext[::-1]}")
        parts.append(np.ascontiguousarray(a).astype(">f8").tobytes())
    Path(path).write_bytes(b"".join(parts))


def _es(v, w=24, d=16):
    """Fortran ES<w>.<d> of a real: one digit before the point, d after, exponent of two digits
    with its E (three digits without it past 99), right-justified in w characters."""
    v = float(v)
    if not math.isfinite(v):
        return f"{'Infinity' if v > 0 else '-Infinity' if v < 0 else 'NaN':>{w}s}"
    m, e = f"{v:.{d}E}".split("E")
    ex = int(e)
    t = f"{m}E{ex:+03d}" if abs(ex) <= 99 else f"{m}{ex:+04d}"
    return f"{t:>{w}s}"


def value_check(name, a):
    """DEBUG_valuecheck's line (mod_misc.f90, format (1x,A,A16,3(A,ES24.16))): max, min and sum
    of an array, the name padded to 16 characters."""
    a = np.asarray(a)
    return f" +check[{name[:16]:<16s}] max={_es(a.max())},min={_es(a.min())},sum={_es(a.sum())}"


def run_snapshot(kernel, path, dims=SnapshotDims(), dt=360.0, device=0, precision="f64", have_sgp=(1,)):
    """Runs the snapshot's inputs through the library and returns (outputs, diffs): the
    computed outputs of the snapshot's region and the poles, and expected - computed per
    output (the driver's point-by-point diff).  precision "f32" runs the FP32 entry points,
    as the drivers built with RP = SP do (they read the same FP64 snapshot and convert)."""
    from icoatmosbenchmark_v1_b200 import api
    if dims.lall != 1:
        raise ValueError("the drivers' snapshots hold one region per process (ADM_lall = 1)")
    if precision not in ("f64", "f32"):
        raise ValueError(f"precision {precision!r}: f64 or f32")
    rp = np.float64 if precision == "f64" else np.float32
    s = read_snapshot(kernel, path, dims)
    # the driver's module globals (problem_size.inc:28-50): one region with the singular point,
    # both poles, levels kmin = 2 .. kmax = kall - 1
    ctx = api.IcoAdv.regions(dims.gall_1d, dims.kall, 2, dims.kall - 1, dims.lall, True, list(have_sgp), device)
    full = {k: np.ascontiguousarray(v) for k, v in s.items()}
    # kernel arguments in the working precision (the metrics stay FP64: the context keeps both).
    # In FP32 the +-HUGE-scale Qout bounds of cells without outflow become +-inf, as the
    # single-precision drivers' conversion of the same snapshot does
    with np.errstate(over="ignore"):
        a = {k: np.ascontiguousarray(v, dtype=rp) for k, v in full.items() if not k.startswith(("GRD_xr", "GMTR_"))}
    try:
        if kernel == "dyn_horiz_adv_flux":
            geo = []
            for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl", "GMTR_a", "GMTR_a_pl"):
                # the library's geometry arrays have no K0 axis: GRD_xr (3, 3, lall, gall) ...
                geo.append(np.ascontiguousarray(np.squeeze(full[k], axis=-2)))
            ctx.set_geometry(*geo)
            # the driver's output arrays start as the snapshot's: points the kernel does not
            # write (the pole centre of flx_h_pl and GRD_xc_pl) keep those values
            flx, flx_pl = a["flx_h"].copy(), a["flx_h_pl"].copy()
            xc, xc_pl = a["GRD_xc"].copy(), a["GRD_xc_pl"].copy()
            ctx.horizontal_flux(flx, flx_pl, xc, xc_pl, a["rho"], a["rho_pl"], a["rhovx"], a["rhovx_pl"],
                                a["rhovy"], a["rhovy_pl"], a["rhovz"], a["rhovz_pl"], float(dt))
            got = OrderedDict(flx_h=flx, flx_h_pl=flx_pl, GRD_xc=xc, GRD_xc_pl=xc_pl)
        elif kernel == "dyn_horiz_adv_limiter":
            qa, qa_pl = a["q_a_prev"].copy(), a["q_a_prev_pl"].copy()
            qo, qo_pl = np.zeros_like(a["Qout_prev"]), np.zeros_like(a["Qout_prev_pl"])
            ctx.horizontal_limiter_thuburn(qa, qa_pl, a["q"], a["q_pl"], a["d"], a["d_pl"], a["ch"], a["ch_pl"],
                                           a["cmask"], a["cmask_pl"], qo, qo_pl, a["Qout_post"], a["Qout_post_pl"])
            got = OrderedDict(q_a=qa, q_a_pl=qa_pl, Qout_prev=qo, Qout_prev_pl=qo_pl)
        else:
            qh, qh_pl = a["q_h_prev"].copy(), a["q_h_prev_pl"].copy()
            ctx.vertical_limiter_thuburn(qh, qh_pl, a["q"], a["q_pl"], a["d"], a["d_pl"], a["ck"], a["ck_pl"])
            got = OrderedDict(q_h=qh, q_h_pl=qh_pl)
    finally:
        ctx.close()
    got = OrderedDict((k, v.astype(np.float64)) for k, v in got.items())
    diffs = OrderedDict((k, s[k] - v) for k, v in got.items())
    return got, diffs


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("action", choices=["check", "run"], help="check: print the arrays' summaries; run: run the "
                    "kernel on the snapshot and print the point-by-point diff")
    ap.add_argument("kernel", choices=KERNELS)
    ap.add_argument("path")
    ap.add_argument("--gall-1d", type=int, default=130)
    ap.add_argument("--kall", type=int, default=42)
    ap.add_argument("--dt", type=float, default=360.0, help="SET_dt_large of the flux driver")
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64",
                    help="f32: the FP32 entry points, as the drivers' single-precision (RP = SP) build")
    a = ap.parse_args(argv)
    dims = SnapshotDims(gall_1d=a.gall_1d, kall=a.kall)
    s = read_snapshot(a.kernel, a.path, dims)
    print(" ### Input ###")
    for k, v in s.items():
        print(value_check(k, v))
    if a.action == "run":
        got, diffs = run_snapshot(a.kernel, a.path, dims, a.dt, precision=a.precision)
        print(" ### Output ###")
        for k, v in got.items():
            print(value_check(k, v))
        print(" ### Validation : point-by-point diff ###")
        for k, v in diffs.items():
            print(value_check("check_" + k, v))


if __name__ == "__main__":
    main()
