"""Region sharding of the batched tracer step across ranks: what each rank sends and receives.

Ranks own contiguous blocks of regions, in the order the reference's region manager hands
them out (communication/src/mod_adm.f90:791-801, RGNMNG_generate_ico), and rank 0 also owns
the two pole centres (mod_adm.f90:190).  A rank runs the step's kernels on its own regions.
Within a step of the batched path one region reads another's values in exactly two places,
and each becomes an exchange between ranks:

1. boundary values (gradient x/y/z, Qout min/max of every tracer and level): a tile reads
   those of the source cell of each of its halo cells, and the seam and pole passes read
   the same; the rank whose boundary pass computed them (the owner of the source cell, or
   rank 0 for a pole centre) sends them;
2. the halo fill of the new state: the copies dst <- src of the composed halo plan
   (COMM_data_transfer, mod_comm.f90:1506-1540) whose two points belong to different ranks.

This module is the host side of that scheme: the index lists of both exchanges for every
pair of ranks, built from the same tables as the single-GPU step (`ica_boundary_tables`,
`ica_comm_plan`).  Points are numbered as in those tables: region points l*gall + ij, then
the 12 pole points lall*gall + 6*p + v.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import api


def region_blocks(nrgn, nranks):
    """Contiguous region ranges [r0, r1) of each rank, the first nrgn % nranks ranks one larger."""
    if nranks < 1 or nranks > nrgn:
        raise ValueError(f"{nranks} ranks for {nrgn} regions")
    base, extra = divmod(nrgn, nranks)
    out, r0 = [], 0
    for r in range(nranks):
        r1 = r0 + base + (1 if r < extra else 0)
        out.append((r0, r1))
        r0 = r1
    return out


@dataclasses.dataclass
class ShardPlan:
    """The exchanges of one step for `nranks` ranks on a glevel/rlevel grid.

    bval_recv[(r, q)]: boundary indices whose values rank r receives from rank q (sorted);
    halo_recv[(r, q)]: (dst, src) point pairs of the halo fill with dst on rank r, src on q;
    halo_local[r]: the pairs with both points on rank r."""
    glevel: int
    rlevel: int
    nranks: int
    blocks: list
    nrgn: int
    gall: int
    blist: np.ndarray
    bval_recv: dict
    halo_recv: dict
    halo_local: dict

    @classmethod
    def build(cls, glevel, rlevel, nranks):
        g1 = 2 ** (glevel - rlevel) + 2
        gall, nrgn = g1 * g1, 10 * 4 ** rlevel
        blocks = region_blocks(nrgn, nranks)
        rank_of_rgn = np.zeros(nrgn, np.int64)
        for r, (a, b) in enumerate(blocks):
            rank_of_rgn[a:b] = r
        npt = nrgn * gall

        def owner(points):
            p = np.asarray(points, np.int64)
            return np.where(p < npt, rank_of_rgn[np.minimum(p, npt - 1) // gall], 0)

        nb, bsrc, blist, ring = api.boundary_tables(glevel, rlevel)
        computed_by = owner(blist)
        bval_recv = {}
        for r, (a, b) in enumerate(blocks):
            need = bsrc[a * gall:b * gall]
            need = need[need >= 0]
            if r == 0:  # the pole pass: its ring slots and the two centres
                need = np.concatenate([need, ring.ravel(), blist.size - 2 + np.arange(2)])
            need = np.unique(need)
            for q in range(nranks):
                if q != r:
                    sel = need[computed_by[need] == q]
                    if sel.size:
                        bval_recv[(r, q)] = sel.astype(np.int32)
        dst, src = api.comm_plan(glevel, rlevel)
        od, os_ = owner(dst), owner(src)
        halo_recv, halo_local = {}, {}
        for r in range(nranks):
            m = od == r
            loc = m & (os_ == r)
            halo_local[r] = (dst[loc], src[loc])
            for q in range(nranks):
                if q != r:
                    sel = m & (os_ == q)
                    if sel.any():
                        halo_recv[(r, q)] = (dst[sel], src[sel])
        return cls(glevel, rlevel, nranks, blocks, nrgn, gall, blist, bval_recv, halo_recv, halo_local)

    def owned_points(self, r):
        """The points rank r computes: its regions' points, and on rank 0 the 12 pole points."""
        a, b = self.blocks[r]
        pts = np.arange(a * self.gall, b * self.gall)
        if r == 0:
            pts = np.concatenate([pts, self.nrgn * self.gall + np.arange(12)])
        return pts

    def bytes_per_step(self, kall, ntr):
        """(boundary-value bytes, halo-fill bytes) sent by every rank together in one step:
        5 FP64 values per tracer and level for a boundary index, rhog and the tracers' rhogq
        per level for a halo point."""
        nb = sum(v.size for v in self.bval_recv.values())
        nh = sum(v[0].size for v in self.halo_recv.values())
        return nb * 5 * 8 * kall * ntr, nh * 8 * kall * (ntr + 1)


# ---- the device side: a rank's part of the step and its two exchanges ------------------------
class LibraryBackend:
    """Pack / unpack of the exchanges with the library's kernels on one context's device buffers
    (ica_shard_bval_pack/unpack, ica_shard_points_pack/unpack): contiguous buffers, no peer access."""

    def __init__(self, ctx):
        self.ctx = ctx

    def pack_bval(self, ntr, kall, bidx):
        import torch
        buf = torch.empty((ntr, kall, bidx.numel(), 5), dtype=torch.float64, device=bidx.device)
        self.ctx.shard_bval(ntr, bidx, buf, unpack=False)
        return buf

    def unpack_bval(self, ntr, kall, bidx, buf):
        self.ctx.shard_bval(ntr, bidx, buf, unpack=True)

    def pack_points(self, pts, var, var_pl):
        import torch
        vmax, kmax = var.shape[0], var.shape[2]
        buf = torch.empty((vmax, kmax, pts.numel()), dtype=torch.float64, device=pts.device)
        self.ctx.shard_points(pts, var, var_pl, buf, unpack=False)
        return buf

    def unpack_points(self, pts, var, var_pl, buf):
        self.ctx.shard_points(pts, var, var_pl, buf, unpack=True)


class TorchBackend:
    """The same pack / unpack as torch index operations on a rank's arrays (any device): the boundary
    values live in `bbuf` (ntr, kall, nb, 5); points index region arrays (vmax, lall, kmax, gall)
    and pole arrays (vmax, 2, kmax, 6) as the flat point numbering does."""

    def __init__(self, bbuf=None):
        self.bbuf = bbuf

    def pack_bval(self, ntr, kall, bidx):
        return self.bbuf[:, :, bidx.long()].clone()

    def unpack_bval(self, ntr, kall, bidx, buf):
        self.bbuf[:, :, bidx.long()] = buf

    @staticmethod
    def _flat(var, var_pl):
        import torch
        m, L, K, G = var.shape
        return torch.cat([var.permute(0, 2, 1, 3).reshape(m, K, L * G), var_pl.permute(0, 2, 1, 3).reshape(m, K, 12)], 2)

    def pack_points(self, pts, var, var_pl):
        return self._flat(var, var_pl)[:, :, pts.long()].contiguous()

    def unpack_points(self, pts, var, var_pl, buf):
        m, L, K, G = var.shape
        f = self._flat(var, var_pl)
        f[:, :, pts.long()] = buf
        var.copy_(f[:, :, :L * G].reshape(m, K, L, G).permute(0, 2, 1, 3))
        var_pl.copy_(f[:, :, L * G:].reshape(m, K, 2, 6).permute(0, 2, 1, 3))


def p2p_exchange(sends, recvs, group=None):
    """One exchange between ranks: sends {q: tensor} to each rank q and receives {q: tensor} (filled
    in place) from each rank q, as one group of point-to-point operations (NCCL send/recv inside
    ncclGroupStart/End on GPUs, gloo on CPUs).  Every rank lists its operations in rank order."""
    import torch.distributed as dist
    ops = []
    for q in sorted(set(sends) | set(recvs)):
        if q in sends:
            ops.append(dist.P2POp(dist.isend, sends[q].contiguous(), q, group=group))
        if q in recvs:
            ops.append(dist.P2POp(dist.irecv, recvs[q], q, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    return recvs


class ShardedRunner:
    """One rank of a region-sharded batched step (ica_shard_set): the rank's part of the step in two
    halves, with the boundary-value exchange between them and the halo exchange of the new state
    after them.  The state is double-buffered (FP64), the fields FP32; every rank holds the whole
    grid's arrays and computes its own regions (and rank 0 the pole centres).

    step() runs the four phases with p2p_exchange over torch.distributed (one process per GPU);
    the phase methods let one process drive several emulated ranks (each with its own context on
    one GPU) and move their buffers itself."""

    def __init__(self, ctx, plan, rank, state, fields, dt, group=None, backend=None):
        import torch
        self.ctx, self.plan, self.rank, self.dt, self.group = ctx, plan, rank, dt, group
        self.backend = backend or LibraryBackend(ctx)
        a0, a1 = plan.blocks[rank]
        dst, src = plan.halo_local[rank]
        ctx.shard_set(a0, a1, rank == 0, dst, src)
        dev = state["rhog"].device
        I = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.int32), device=dev)  # noqa: E731
        self.bsend = {q: I(v) for (r, q2), v in plan.bval_recv.items() if q2 == rank for q in [r]}
        self.brecv = {q: I(v) for (r, q), v in plan.bval_recv.items() if r == rank}
        self.hsend = {q: I(v[1]) for (r, q2), v in plan.halo_recv.items() if q2 == rank for q in [r]}
        self.hrecv = {q: I(v[0]) for (r, q), v in plan.halo_recv.items() if r == rank}
        self.a = state
        self.b = {k: torch.empty_like(v) for k, v in state.items()}
        from .api import FIELD_KEYS
        self.f32 = {k: fields[k].to(torch.float32).contiguous() for k in FIELD_KEYS}
        self.ntr = int(state["rhogq"].shape[0])
        self.kall = int(state["rhog"].shape[1])

    @property
    def state(self):
        return self.a

    # ---- phases
    def part(self, p):
        self.ctx.advect_fast_part_dev(p, self.dt, self.a, self.b, self.f32)

    def bval_sends(self):
        return {q: self.backend.pack_bval(self.ntr, self.kall, idx) for q, idx in self.bsend.items()}

    def bval_recv_buffers(self):
        import torch
        dev = self.a["rhog"].device
        return {q: torch.empty((self.ntr, self.kall, idx.numel(), 5), dtype=torch.float64, device=dev)
                for q, idx in self.brecv.items()}

    def bval_unpack(self, bufs):
        for q, buf in bufs.items():
            self.backend.unpack_bval(self.ntr, self.kall, self.brecv[q], buf)

    def _state_vars(self, S):
        return ((S["rhog"].unsqueeze(0), S["rhog_pl"].unsqueeze(0)), (S["rhogq"], S["rhogq_pl"]))

    def halo_sends(self):
        import torch
        out = {}
        for q, pts in self.hsend.items():
            out[q] = torch.cat([self.backend.pack_points(pts, v, vp) for v, vp in self._state_vars(self.b)], 0)
        return out

    def halo_recv_buffers(self):
        import torch
        dev = self.a["rhog"].device
        return {q: torch.empty((1 + self.ntr, self.kall, pts.numel()), dtype=torch.float64, device=dev)
                for q, pts in self.hrecv.items()}

    def halo_unpack(self, bufs):
        for q, buf in bufs.items():
            (r, rp), (t, tp) = self._state_vars(self.b)
            self.backend.unpack_points(self.hrecv[q], r, rp, buf[:1])
            self.backend.unpack_points(self.hrecv[q], t, tp, buf[1:])

    def swap(self):
        self.a, self.b = self.b, self.a

    def step(self):
        self.part(1)
        self.bval_unpack(p2p_exchange(self.bval_sends(), self.bval_recv_buffers(), self.group))
        self.part(2)
        self.halo_unpack(p2p_exchange(self.halo_sends(), self.halo_recv_buffers(), self.group))
        self.swap()


def emulated_step(runners):
    """One step of several ranks driven by one process (one GPU, a context per rank): each phase
    runs on every rank before the next, and the exchanges copy each sender's packed buffer into
    the receiver's buffer.  No kernel of one rank waits for another's."""
    for r in runners:
        r.part(1)
    sends = [r.bval_sends() for r in runners]
    for r in runners:
        bufs = r.bval_recv_buffers()
        for q, buf in bufs.items():
            buf.copy_(sends[q][r.rank])
        r.bval_unpack(bufs)
    for r in runners:
        r.part(2)
    sends = [r.halo_sends() for r in runners]
    for r in runners:
        bufs = r.halo_recv_buffers()
        for q, buf in bufs.items():
            buf.copy_(sends[q][r.rank])
        r.halo_unpack(bufs)
    for r in runners:
        r.swap()
