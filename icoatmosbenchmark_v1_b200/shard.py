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
