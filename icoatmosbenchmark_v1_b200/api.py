"""Python host interface over libicoadv.so (the C ABI in include/icoadv.h).

Method names, argument order and meaning follow the reference subroutines:

    horizontal_flux            kernels/NICAM/dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-49
    horizontal_limiter_thuburn kernels/NICAM/dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-49
    vertical_limiter_thuburn   kernels/NICAM/dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-45
    COMM_data_transfer         kernels/NICAM/communication/src/mod_comm.f90:1506-1508
    COMM_var                   kernels/NICAM/communication/src/mod_comm.f90:1895-1899

Arrays are numpy (host) or torch CUDA tensors (device), C-contiguous, in the
reference's Fortran layout written in C order: var(gall,kall,lall,m) has
shape (m, lall, kall, gall).  Host arrays go through the host-pointer entry
points (copy in, run, copy out); CUDA tensors go through the *_dev entry
points on the context's stream, ordered after the work already queued on
torch's current stream and before anything queued there afterwards (event
waits, no host synchronisation), so tensors can be handed back and forth
with torch without explicit synchronisation.  Errors raise IcoAdvError with the library's
message.  There is no CPU fallback: without the built library or a B200 the
calls fail.
"""
from __future__ import annotations

import contextlib
import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libicoadv.so"
_lib = None

ICA_OK = 0
ERRORS = {-1: "ICA_ERR_ARG", -2: "ICA_ERR_STATE", -3: "ICA_ERR_CUDA", -4: "ICA_ERR_TIMEOUT",
          -5: "ICA_ERR_INTERNAL", -6: "ICA_ERR_NOMEM"}


class IcoAdvError(RuntimeError):
    def __init__(self, fn, rc):
        self.rc = rc
        super().__init__(f"{fn} failed: {ERRORS.get(rc, rc)}: {lib().ica_last_error().decode()}")


class Dims(C.Structure):
    _fields_ = [("glevel", C.c_int), ("rlevel", C.c_int), ("vlayer", C.c_int), ("device", C.c_int)]


class Sizes(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("gall_1d", "gall", "gmin", "gmax", "kall", "kmin", "kmax",
                                       "lall", "gall_pl", "lall_pl")]


def lib():
    """Loads libicoadv.so (built in-tree by icoatmosbenchmark_v1_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run icoatmosbenchmark_v1_b200.build.build()")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.ica_last_error.restype = C.c_char_p
        _lib.ica_stream.restype = C.c_void_p
        _lib.ica_stream.argtypes = [C.c_void_p]
        _lib.ica_launch_count.restype = C.c_longlong
        _lib.ica_launch_count.argtypes = [C.c_void_p]
        _lib.ica_init.argtypes = [C.POINTER(Dims), C.POINTER(C.c_void_p)]
        _lib.ica_finalize.argtypes = [C.c_void_p]
        _lib.ica_get_sizes.argtypes = [C.c_void_p, C.POINTER(Sizes)]
    return _lib


def exported_symbols():
    """Names of the functions declared in include/icoadv.h."""
    import re
    text = (PKG.parent / "include" / "icoadv.h").read_text()
    return sorted(set(re.findall(r"^(?:int|void|const char|long long)[\s*]+(ica_\w+)\s*\(", text, re.M)))


def _check(fn, rc):
    if rc != ICA_OK:
        raise IcoAdvError(fn, rc)


# ---- host-only topology helpers ------------------------------------------------
def comm_plan(glevel, rlevel, pole_fill=False):
    """Composed single-process halo fill: arrays (dst, src) of point indices."""
    n = C.c_int(0)
    _check("ica_comm_plan", lib().ica_comm_plan(glevel, rlevel, int(pole_fill), C.byref(n), None, None))
    dst = np.zeros(n.value, np.int32)
    src = np.zeros(n.value, np.int32)
    _check("ica_comm_plan", lib().ica_comm_plan(glevel, rlevel, int(pole_fill), C.byref(n),
                                                dst.ctypes.data_as(C.POINTER(C.c_int)),
                                                src.ctypes.data_as(C.POINTER(C.c_int))))
    return dst, src


def topology_info(glevel, rlevel):
    nr = 10 * 4 ** rlevel
    sgp = np.zeros(nr, np.int32)
    r4 = np.zeros(2, np.int32)
    ring = np.zeros((2, 5), np.int32)
    ip = C.POINTER(C.c_int)
    _check("ica_topology_info", lib().ica_topology_info(glevel, rlevel, sgp.ctypes.data_as(ip),
                                                        r4.ctypes.data_as(ip), ring.ctypes.data_as(ip)))
    return sgp, r4, ring


def boundary_tables(glevel, rlevel):
    """The batched step's boundary-value tables (ica_boundary_tables): nb, bsrc (lall*gall),
    blist (nb), pole_ring (2, 5)."""
    nb = C.c_int(0)
    ip = C.POINTER(C.c_int)
    _check("ica_boundary_tables", lib().ica_boundary_tables(glevel, rlevel, C.byref(nb), None, None, None))
    g1 = 2 ** (glevel - rlevel) + 2
    bsrc = np.zeros(10 * 4 ** rlevel * g1 * g1, np.int32)
    blist = np.zeros(nb.value, np.int32)
    ring = np.zeros((2, 5), np.int32)
    _check("ica_boundary_tables", lib().ica_boundary_tables(glevel, rlevel, C.byref(nb), bsrc.ctypes.data_as(ip),
                                                            blist.ctypes.data_as(ip), ring.ctypes.data_as(ip)))
    return nb.value, bsrc, blist, ring


def apply_plan_numpy(plan, var, var_pl):
    """Host-side application of a plan (used to fill halos of synthetic inputs)."""
    from .grid import apply_plan_numpy as apply
    apply(plan, var, var_pl)


# ---- the context ------------------------------------------------------------------
def _ptr(a, want):
    """Pointer of a numpy array (host) or a torch CUDA tensor (device)."""
    if a is None:
        return None, None
    if isinstance(a, np.ndarray):
        if a.dtype != want or not a.flags.c_contiguous:
            raise TypeError(f"expected C-contiguous {want} array, got {a.dtype}")
        return a.ctypes.data_as(C.c_void_p), False
    try:
        import torch
    except ImportError:  # pragma: no cover
        raise TypeError("unsupported array type")
    if isinstance(a, torch.Tensor):
        tw = {np.float64: torch.float64, np.float32: torch.float32}[np.dtype(want).type]
        if a.dtype != tw or not a.is_contiguous() or not a.is_cuda:
            raise TypeError(f"expected contiguous CUDA tensor of {tw}, got {a.dtype} on {a.device}")
        return C.c_void_p(a.data_ptr()), True
    raise TypeError(f"unsupported array type {type(a)}")


class IcoAdv:
    """One grid on one GPU: ADM sizes, metrics, halo plan and a CUDA stream."""

    def __init__(self, glevel, rlevel, vlayer, device=0):
        self.h = C.c_void_p()
        d = Dims(glevel, rlevel, vlayer, device)
        _check("ica_init", lib().ica_init(C.byref(d), C.byref(self.h)))
        s = Sizes()
        _check("ica_get_sizes", lib().ica_get_sizes(self.h, C.byref(s)))
        self.sizes = s
        self.glevel, self.rlevel, self.vlayer, self.device = glevel, rlevel, vlayer, device
        self._ext = None

    @classmethod
    def regions(cls, gall_1d, kall, kmin, kmax, lall, have_pl, have_sgp, device=0):
        """A context for arrays that hold part of a grid, sized as a reference kernel driver
        holds them (ADM_gall_1d, ADM_kall, ADM_kmin, ADM_kmax, ADM_lall, ADM_have_pl,
        ADM_have_sgp): ica_init_regions.  It has no region topology (no halo fill)."""
        self = cls.__new__(cls)
        self.h = C.c_void_p()
        sg = np.ascontiguousarray(np.asarray(have_sgp, dtype=np.int32).reshape(-1))
        if sg.size != lall:
            raise ValueError("have_sgp needs lall entries")
        _check("ica_init_regions", lib().ica_init_regions(int(gall_1d), int(kall), int(kmin), int(kmax), int(lall),
                                                          int(bool(have_pl)), sg.ctypes.data_as(C.POINTER(C.c_int)),
                                                          int(device), C.byref(self.h)))
        s = Sizes()
        _check("ica_get_sizes", lib().ica_get_sizes(self.h, C.byref(s)))
        self.sizes = s
        self.glevel = self.rlevel = None
        self.vlayer, self.device = kall - 2, device
        self._ext = None
        return self

    def close(self):
        if self.h:
            lib().ica_finalize(self.h)
            self.h = C.c_void_p()
            self._ext = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().ica_stream(self.h)

    @contextlib.contextmanager
    def _ordered(self, dev=True):
        """Stream order of a device call against torch's current stream: the context
        stream waits for what torch queued before it, torch waits for the call."""
        if not dev:
            yield
            return
        import torch
        if self._ext is None:
            self._ext = torch.cuda.ExternalStream(self.stream, device=self.device)
        cur = torch.cuda.current_stream(self.device)
        self._ext.wait_stream(cur)
        yield
        cur.wait_stream(self._ext)

    @property
    def launch_count(self):
        return lib().ica_launch_count(self.h)

    def set_geometry(self, GRD_xr, GRD_xr_pl, GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl):
        keep = [np.ascontiguousarray(a, np.float64)
                for a in (GRD_xr, GRD_xr_pl, GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl)]
        _check("ica_set_geometry", lib().ica_set_geometry(self.h, *[_ptr(a, np.float64)[0] for a in keep]))

    def _call(self, name, dtype, arrays, *scalars):
        ptrs, kinds = zip(*[_ptr(a, dtype) for a in arrays])
        dev = {k for k in kinds if k is not None}
        if len(dev) != 1:
            raise TypeError("mix of host and device arrays")
        dev = dev.pop()
        suffix = "_dev" if dev else ""
        if dtype == np.float32:
            if dev:
                raise TypeError(f"{name}: FP32 entry points take host arrays")
            suffix = "_f32"
        fn = getattr(lib(), name + suffix)
        with self._ordered(dev):
            _check(name + suffix, fn(self.h, *ptrs, *scalars))

    @staticmethod
    def _dtype(a):
        if isinstance(a, np.ndarray):
            return a.dtype.type
        import torch
        return {torch.float64: np.float64, torch.float32: np.float32}[a.dtype]

    def horizontal_flux(self, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, rhovx, rhovx_pl,
                        rhovy, rhovy_pl, rhovz, rhovz_pl, dt):
        t = self._dtype(rho)
        sc = C.c_double(dt) if t == np.float64 else C.c_float(dt)
        self._call("ica_horizontal_flux", t, [flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, rhovx, rhovx_pl,
                                              rhovy, rhovy_pl, rhovz, rhovz_pl], sc)

    def horizontal_limiter_thuburn(self, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl,
                                   Qout_prev, Qout_prev_pl, Qout_post=None, Qout_post_pl=None):
        t = self._dtype(q)
        arrs = [q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl, Qout_prev, Qout_prev_pl]
        ptrs, kinds = zip(*[_ptr(a, t) for a in arrs])
        post = [_ptr(Qout_post, t)[0], _ptr(Qout_post_pl, t)[0]]
        dev = kinds[0]
        name = "ica_horizontal_limiter_thuburn" + ("_dev" if dev else ("_f32" if t == np.float32 else ""))
        with self._ordered(dev):
            _check(name, getattr(lib(), name)(self.h, *ptrs, *post))

    def vertical_limiter_thuburn(self, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl):
        self._call("ica_vertical_limiter_thuburn", self._dtype(q), [q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl])

    def COMM_data_transfer(self, var, var_pl):
        vmax, _, kmax, _ = var.shape
        self._call("ica_comm_data_transfer", self._dtype(var), [var, var_pl], int(kmax), int(vmax))

    def COMM_var(self, var, var_pl):
        vmax, _, kmax, _ = var.shape
        self._call("ica_comm_var", self._dtype(var), [var, var_pl], int(kmax), int(vmax))

    # ---- composed step -----------------------------------------------------------
    GRID_KEYS = (("GRD_x", (3,), (3, 2, 6)), ("GRD_xr", (3, 3), (3, 2, 6)), ("GMTR_p", (8,), (8, 2, 6)),
                 ("GMTR_t", (5, 2), (5, 2, 6)), ("GMTR_a", (12, 3), (18, 2, 6)))

    def build_grid(self, radius):
        """The grid's positions and metrics built on the device (ica_grid_build_dev): a dict of
        CUDA tensors with the names and shapes of grid.Grid.arrays (GRD_x, GRD_xr, GMTR_p/t/a,
        coef_grad and their pole arrays)."""
        import torch
        L, g = self.sizes.lall, self.sizes.gall
        dev = torch.device("cuda", self.device)
        out = {}
        for name, lead, pl in self.GRID_KEYS:
            out[name] = torch.empty(lead + (L, g), dtype=torch.float64, device=dev)
            out[name + "_pl"] = torch.empty(pl, dtype=torch.float64, device=dev)
        out["coef_grad"] = torch.empty((L, 3, 7, g), dtype=torch.float64, device=dev)
        out["coef_grad_pl"] = torch.empty((2, 3, 6), dtype=torch.float64, device=dev)
        order = ("GRD_x", "GRD_x_pl", "GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                 "GMTR_a", "GMTR_a_pl", "coef_grad", "coef_grad_pl")
        with self._ordered():
            _check("ica_grid_build_dev", lib().ica_grid_build_dev(self.h, C.c_double(radius),
                                                                  *[C.c_void_p(out[k].data_ptr()) for k in order]))
        return out

    def set_step_geometry(self, GRD_x, GRD_x_pl, coef_grad, coef_grad_pl, rdgz, afact, bfact):
        keep = [np.ascontiguousarray(a, np.float64) for a in (GRD_x, GRD_x_pl, coef_grad, coef_grad_pl, rdgz, afact,
                                                               bfact)]
        _check("ica_set_step_geometry", lib().ica_set_step_geometry(self.h, *[_ptr(a, np.float64)[0] for a in keep]))

    def set_grid(self, grid):
        """Registers the metrics and step geometry of an icoatmosbenchmark_v1_b200.grid.Grid."""
        A = grid.arrays
        self.set_geometry(*[A[k] for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                                           "GMTR_a", "GMTR_a_pl")])
        self.set_step_geometry(A["GRD_x"], A["GRD_x_pl"], A["coef_grad"], A["coef_grad_pl"], A["rdgz"], A["afact"],
                               A["bfact"])

    def advect_step(self, dt, rhog, rhog_pl, rhogq, rhogq_pl, rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz,
                    rhogvz_pl, rhogw, rhogw_pl):
        """One composed FP64 step in place (plain per-tracer path)."""
        ntr = rhogq.shape[0]
        arrs = [rhog, rhog_pl, rhogq, rhogq_pl, rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz, rhogvz_pl, rhogw, rhogw_pl]
        ptrs, kinds = zip(*[_ptr(a, np.float64) for a in arrs])
        name = "ica_advect_step" + ("_dev" if kinds[0] else "")
        with self._ordered(bool(kinds[0])):
            _check(name, getattr(lib(), name)(self.h, int(ntr), C.c_double(dt), *ptrs))

    # ---- adjoint of the plain step ---------------------------------------------------
    def advect_step_adjoint(self, dt, state, fields, a_state, a_wind):
        """Reverse mode of one plain FP64 step.  state / fields: dicts (STATE_KEYS, FIELD_KEYS)
        of the step's input (unchanged); a_state (STATE_KEYS): adjoint of the step's output
        on entry, of its input on return; a_wind (WIND_KEYS): accumulated.  All numpy
        (host) or all CUDA tensors (device)."""
        ntr = state["rhogq"].shape[0]
        arrs = ([state[k] for k in STATE_KEYS] + [fields[k] for k in FIELD_KEYS] + [a_state[k] for k in STATE_KEYS]
                + [a_wind[k] for k in WIND_KEYS])
        ptrs, kinds = zip(*[_ptr(a, np.float64) for a in arrs])
        if len(set(kinds)) != 1:
            raise TypeError("mix of host and device arrays")
        name = "ica_advect_step_adjoint" + ("_dev" if kinds[0] else "")
        with self._ordered(bool(kinds[0])):
            _check(name, getattr(lib(), name)(self.h, int(ntr), C.c_double(dt), *ptrs))

    def adjoint_record(self, dt, nsteps, every, state, fields):
        """Advances the device state nsteps plain FP64 steps in place, keeping a checkpoint
        every `every` steps for adjoint_sweep."""
        ntr = state["rhogq"].shape[0]
        sp = [_ptr(state[k], np.float64)[0] for k in STATE_KEYS]
        fp = [_ptr(fields[k], np.float64)[0] for k in FIELD_KEYS]
        with self._ordered():
            _check("ica_adjoint_record", lib().ica_adjoint_record(self.h, int(ntr), C.c_double(dt), int(nsteps),
                                                                  int(every), *sp, *fp))

    def adjoint_sweep(self, fields, a_state, a_wind):
        """Adjoint of the recorded run: a_state holds the adjoint of the final state on entry
        and of the initial state on return; a_wind is accumulated (device tensors)."""
        fp = [_ptr(fields[k], np.float64)[0] for k in FIELD_KEYS]
        ap = [_ptr(a_state[k], np.float64)[0] for k in STATE_KEYS] + [_ptr(a_wind[k], np.float64)[0]
                                                                      for k in WIND_KEYS]
        with self._ordered():
            _check("ica_adjoint_sweep", lib().ica_adjoint_sweep(self.h, *fp, *ap))

    def adjoint_release(self):
        _check("ica_adjoint_release", lib().ica_adjoint_release(self.h))

    # ---- batched path (all tracers per launch) -------------------------------------
    def advect_fast_dev(self, dt, state_in, state_out, fields32):
        """One batched step on device tensors: state dicts (rhog, rhog_pl, rhogq, rhogq_pl) FP64,
        fields32 dict (rhogvx..rhogw_pl) FP32; writes state_out."""
        ntr = state_in["rhogq"].shape[0]
        sp = [_ptr(state_in[k], np.float64)[0] for k in STATE_KEYS]
        so = [_ptr(state_out[k], np.float64)[0] for k in STATE_KEYS]
        fp = [_ptr(fields32[k], np.float32)[0] for k in FIELD_KEYS]
        with self._ordered():
            _check("ica_advect_fast_dev", lib().ica_advect_fast_dev(self.h, int(ntr), C.c_double(dt), *sp, *so,
                                                                    *fp))

    def advect_fast64_dev(self, dt, state_in, state_out, fields64):
        """The FP64 variant of the batched step (FP64 fields, FP64 faces and limiters)."""
        ntr = state_in["rhogq"].shape[0]
        sp = [_ptr(state_in[k], np.float64)[0] for k in STATE_KEYS]
        so = [_ptr(state_out[k], np.float64)[0] for k in STATE_KEYS]
        fp = [_ptr(fields64[k], np.float64)[0] for k in FIELD_KEYS]
        with self._ordered():
            _check("ica_advect_fast64_dev", lib().ica_advect_fast64_dev(self.h, int(ntr), C.c_double(dt), *sp, *so,
                                                                        *fp))

    def advect_fast_host(self, dt, rhog, rhog_pl, rhogq, rhogq_pl, rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz,
                         rhogvz_pl, rhogw, rhogw_pl):
        """One batched step on host arrays, in place on the FP64 state (FP32 fields)."""
        ntr = rhogq.shape[0]
        sp = [_ptr(a, np.float64)[0] for a in (rhog, rhog_pl, rhogq, rhogq_pl)]
        fp = [_ptr(a, np.float32)[0] for a in (rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz, rhogvz_pl, rhogw,
                                             rhogw_pl)]
        _check("ica_advect_fast", lib().ica_advect_fast(self.h, int(ntr), C.c_double(dt), *sp, *fp))

    def advect_fast_part_dev(self, part, dt, state_in, state_out, fields32):
        """Half of a batched step of a region-sharded rank: part 1 the boundary pass, part 2 the
        rest and the rank's own halo copies (ica_advect_fast_part_dev)."""
        ntr = state_in["rhogq"].shape[0]
        sp = [_ptr(state_in[k], np.float64)[0] for k in STATE_KEYS]
        so = [_ptr(state_out[k], np.float64)[0] for k in STATE_KEYS]
        fp = [_ptr(fields32[k], np.float32)[0] for k in FIELD_KEYS]
        with self._ordered():
            _check("ica_advect_fast_part_dev", lib().ica_advect_fast_part_dev(self.h, int(part), int(ntr),
                                                                              C.c_double(dt), *sp, *so, *fp))

    def shard_set(self, l0, l1, poles, dst=None, src=None):
        """This context computes regions [l0, l1) (and the pole centres if poles), with the halo
        copies dst <- src whose two points it owns; shard_set(None, ...) returns to the whole grid."""
        if l0 is None:
            _check("ica_shard_set", lib().ica_shard_set(self.h, 0, 0, 0, -1, None, None))
            return
        d = np.ascontiguousarray(dst, np.int32)
        s = np.ascontiguousarray(src, np.int32)
        ip = C.POINTER(C.c_int)
        _check("ica_shard_set", lib().ica_shard_set(self.h, int(l0), int(l1), int(bool(poles)), int(d.size),
                                                    d.ctypes.data_as(ip), s.ctypes.data_as(ip)))

    def shard_bval(self, ntr, bidx, buf, unpack):
        fn = lib().ica_shard_bval_unpack if unpack else lib().ica_shard_bval_pack
        with self._ordered():
            _check("ica_shard_bval", fn(self.h, int(ntr), int(bidx.numel()), C.c_void_p(bidx.data_ptr()),
                                        C.c_void_p(buf.data_ptr())))

    def shard_points(self, pts, var, var_pl, buf, unpack):
        fn = lib().ica_shard_points_unpack if unpack else lib().ica_shard_points_pack
        vmax, kmax = int(var.shape[0]), int(var.shape[2])
        with self._ordered():
            _check("ica_shard_points", fn(self.h, int(pts.numel()), C.c_void_p(pts.data_ptr()), kmax, vmax,
                                          C.c_void_p(var.data_ptr()), C.c_void_p(var_pl.data_ptr()),
                                          C.c_void_p(buf.data_ptr())))

    def fast_shapes(self):
        n = C.c_int()
        _check("ica_fast_shapes", lib().ica_fast_shapes(self.h, C.byref(n), None, None, None))
        tx, ty, tg = (np.zeros(n.value, np.int32) for _ in range(3))
        ip = C.POINTER(C.c_int)
        _check("ica_fast_shapes", lib().ica_fast_shapes(self.h, C.byref(n), tx.ctypes.data_as(ip),
                                                        ty.ctypes.data_as(ip), tg.ctypes.data_as(ip)))
        return list(zip(tx.tolist(), ty.tolist(), tg.tolist()))

    def fast_set_shape(self, shape):
        _check("ica_fast_set_shape", lib().ica_fast_set_shape(self.h, int(shape)))

    def fast_set_host_chunk(self, tracers):
        """Tracers per chunk of advect_fast_host's overlapped copies (0: by size)."""
        _check("ica_fast_set_host_chunk", lib().ica_fast_set_host_chunk(self.h, int(tracers)))

    def fast_status(self):
        """Status word of the batched kernels since the last call (0: every bounded wait of
        the horizontal kernel ended in time); reading it clears it."""
        f = C.c_int(0)
        rc = lib().ica_fast_status(self.h, C.byref(f))
        if rc not in (0, -4):
            _check("ica_fast_status", rc)
        return f.value

    def fast_timing(self, enable):
        ms = C.c_double()
        n = C.c_longlong()
        _check("ica_fast_timing", lib().ica_fast_timing(self.h, int(enable), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def fast_runner(self, grid, state, fields, dt, autotune=True, f64=False):
        return FastRunner(self, grid, state, fields, dt, autotune, f64)


STATE_KEYS = ("rhog", "rhog_pl", "rhogq", "rhogq_pl")
FIELD_KEYS = ("rhogvx", "rhogvx_pl", "rhogvy", "rhogvy_pl", "rhogvz", "rhogvz_pl", "rhogw", "rhogw_pl")
WIND_KEYS = ("rhogvx", "rhogvx_pl", "rhogvy", "rhogvy_pl", "rhogvz", "rhogvz_pl")


class FastRunner:
    """Device-resident loop of the batched step: double-buffered FP64 state, FP32 fields (FP64
    fields and arithmetic for the FP64 variant, f64=True), tile shape chosen by timing every
    available shape on the real inputs (the autotuner)."""

    def __init__(self, ctx, grid, state, fields, dt, autotune=True, f64=False):
        import torch
        self.ctx, self.dt = ctx, dt
        self.f64 = bool(f64)
        self.a = state
        self.b = {k: torch.empty_like(v) for k, v in state.items()}
        ft = torch.float64 if self.f64 else torch.float32
        self.f32 = {k: fields[k].to(ft).contiguous() for k in FIELD_KEYS}
        self.updates = (10 * 4 ** grid.glevel + 2) * grid.kall * state["rhogq"].shape[0]
        # algorithmic bytes of one tracer cell-level update: rhogq read + write (FP64); per cell-level,
        # shared by the tracers: rhog old and new (FP64) and rhogv x/y/z + rhogw (FP32, or FP64)
        self.alg_bytes = 16.0 + (48.0 if self.f64 else 32.0) / state["rhogq"].shape[0]
        self.shape = 0
        self.tuning = []
        if autotune:
            self.autotune()

    @property
    def state(self):
        return self.a

    def step(self):
        if self.f64:
            self.ctx.advect_fast64_dev(self.dt, self.a, self.b, self.f32)
        else:
            self.ctx.advect_fast_dev(self.dt, self.a, self.b, self.f32)
        self.a, self.b = self.b, self.a

    def autotune(self, reps=2):
        import torch
        shapes = self.ctx.fast_shapes()
        saved = {k: v.clone() for k, v in self.a.items()}
        best = None
        for s in range(len(shapes)):
            self.ctx.fast_set_shape(s)
            self.step()
            self.ctx.fast_timing(1)
            for _ in range(reps):
                self.step()
            ms, n = self.ctx.fast_timing(0)
            t = ms / max(n, 1)
            self.tuning.append({"shape": shapes[s], "ms": t})
            if best is None or t < best[1]:
                best = (s, t)
        self.shape = best[0]
        self.ctx.fast_set_shape(self.shape)
        for k in self.a:
            self.a[k].copy_(saved[k])
        torch.cuda.synchronize()

    def start_timing(self):
        self.ctx.fast_timing(1)

    def kernel_stats(self):
        """Average CUDA-event duration of the horizontal sub-step (the face-flux prologue
        k_fast_faces and the tile kernel k_fast_horiz, timed together) over the steps since
        start_timing()."""
        ms, n = self.ctx.fast_timing(0)
        if n == 0:
            return None
        return {"name": "k_fast_faces+k_fast_horiz", "ms_per_launch": ms / n, "launches": n,
                "bytes_per_launch": self.updates * self.alg_bytes}


# ---- batches of grid instances (uneven grid levels) ------------------------------
class FastArgs(C.Structure):
    """ica_fast_args: one instance's step arguments (device pointers)."""
    _fields_ = [("ntr", C.c_int), ("dt", C.c_double)] + [
        (n, C.c_void_p) for n in ("rhog_in", "rhog_in_pl", "rhogq_in", "rhogq_in_pl", "rhog_out", "rhog_out_pl",
                                  "rhogq_out", "rhogq_out_pl") + FIELD_KEYS]


def _fast_args(dt, state_in, state_out, fields32):
    a = FastArgs()
    a.ntr, a.dt = int(state_in["rhogq"].shape[0]), float(dt)
    for k, kin, kout in (("rhog", "rhog_in", "rhog_out"), ("rhog_pl", "rhog_in_pl", "rhog_out_pl"),
                         ("rhogq", "rhogq_in", "rhogq_out"), ("rhogq_pl", "rhogq_in_pl", "rhogq_out_pl")):
        setattr(a, kin, state_in[k].data_ptr())
        setattr(a, kout, state_out[k].data_ptr())
    for k in FIELD_KEYS:
        setattr(a, k, fields32[k].data_ptr())
    return a


class Batch:
    """Several grid instances (each an IcoAdv context with its geometry) advanced by the same
    launches (ica_batch_*): one launch per stage over all instances, the horizontal kernel
    persistent; a step can be captured in a CUDA graph and replayed."""

    def __init__(self, ctxs):
        self.ctxs = list(ctxs)
        self.h = C.c_void_p()
        arr = (C.c_void_p * len(self.ctxs))(*[c.h.value for c in self.ctxs])
        _check("ica_batch_create", lib().ica_batch_create(arr, len(self.ctxs), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().ica_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, shape):
        _check("ica_batch_set_shape", lib().ica_batch_set_shape(self.h, int(shape)))

    def _args(self, args):
        return (FastArgs * len(args))(*args)

    def step(self, args, f64=False):
        """One step of every instance; f64: the FP64 variant (args with FP64 fields)."""
        name = "ica_batch_step64_dev" if f64 else "ica_batch_step_dev"
        with self.ctxs[0]._ordered():
            _check(name, getattr(lib(), name)(self.h, self._args(args)))

    def capture(self, args, slot, f64=False):
        name = "ica_batch_capture64" if f64 else "ica_batch_capture"
        _check(name, getattr(lib(), name)(self.h, self._args(args), int(slot)))

    def replay(self, slot):
        with self.ctxs[0]._ordered():
            _check("ica_batch_replay", lib().ica_batch_replay(self.h, int(slot)))


class BatchRunner:
    """Device-resident loop over a batch of instances: per instance a double-buffered FP64
    state and FP32 fields (FP64 fields for the FP64 variant, f64=True); step() launches
    directly, or, after use_graph(), replays the captured CUDA graph of the current direction."""

    def __init__(self, ctxs, states, fields, dts, shape=0, f64=False):
        import torch
        self.batch = Batch(ctxs)
        self.batch.set_shape(shape)
        self.f64 = bool(f64)
        self.a = list(states)
        self.b = [{k: torch.empty_like(v) for k, v in s.items()} for s in states]
        ft = torch.float64 if self.f64 else torch.float32
        self.f32 = [{k: f[k].to(ft).contiguous() for k in FIELD_KEYS} for f in fields]
        self.dts = list(dts)
        self.graphs = False
        self.parity = 0  # 0: a -> b next, 1: b -> a next
        # tracer cell-level updates per step: columns (10 * 4^glevel + 2) x kall x tracers
        self.updates = sum((10 * 4 ** c.glevel + 2) * int(s["rhogq"].shape[2]) * int(s["rhogq"].shape[0])
                           for c, s in zip(ctxs, states))

    def _argsets(self):
        fwd = [_fast_args(dt, a, b, f) for dt, a, b, f in zip(self.dts, self.a, self.b, self.f32)]
        bwd = [_fast_args(dt, b, a, f) for dt, a, b, f in zip(self.dts, self.a, self.b, self.f32)]
        return fwd, bwd

    @property
    def states(self):
        return self.a if self.parity == 0 else self.b

    def step(self):
        if self.graphs:
            self.batch.replay(self.parity)
        else:
            self.batch.step(self._argsets()[self.parity], self.f64)
        self.parity ^= 1

    def use_graph(self):
        """Capture both directions (after one uncaptured step has set up every buffer)."""
        fwd, bwd = self._argsets()
        self.batch.capture(fwd, 0, self.f64)
        self.batch.capture(bwd, 1, self.f64)
        self.graphs = True

    def close(self):
        self.batch.close()
