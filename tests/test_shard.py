"""The host side of region sharding (icoatmosbenchmark_v1_b200.shard): the plan's lists cover
every value a rank reads from another rank exactly once, and two gloo ranks that exchange
along them end with the halos of the single-process fill.  Packing and unpacking are numpy
gathers here; on GPUs they are the library's pack/unpack step around NCCL send/recv."""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def plans(built):
    from icoatmosbenchmark_v1_b200 import shard
    return {(g, rl, n): shard.ShardPlan.build(g, rl, n) for g, rl, n in
            [(4, 0, 1), (4, 0, 2), (4, 0, 3), (4, 1, 4), (4, 1, 7), (5, 0, 10)]}


def test_region_blocks():
    from icoatmosbenchmark_v1_b200.shard import region_blocks
    assert region_blocks(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert region_blocks(40, 8) == [(5 * r, 5 * r + 5) for r in range(8)]
    with pytest.raises(ValueError):
        region_blocks(10, 11)


def test_single_rank_plan_is_local(plans):
    from icoatmosbenchmark_v1_b200 import api
    p = plans[(4, 0, 1)]
    assert not p.bval_recv and not p.halo_recv
    dst, src = api.comm_plan(4, 0)
    np.testing.assert_array_equal(p.halo_local[0][0], dst)
    np.testing.assert_array_equal(p.halo_local[0][1], src)


@pytest.mark.parametrize("key", [(4, 0, 2), (4, 0, 3), (4, 1, 4), (4, 1, 7), (5, 0, 10)])
def test_plan_covers_every_read_once(plans, key):
    from icoatmosbenchmark_v1_b200 import api
    p = plans[key]
    g, rl, n = key
    dst, src = api.comm_plan(g, rl)
    nb, bsrc, blist, ring = api.boundary_tables(g, rl)
    npt = p.nrgn * p.gall

    def owner(pt):
        return 0 if pt >= npt else next(r for r, (a, b) in enumerate(p.blocks) if a <= pt // p.gall < b)

    # halo fill: every plan copy appears once, on the rank of its destination, local or
    # received from the rank of its source
    seen = {}
    for r in range(n):
        pairs = [p.halo_local[r]] + [v for (rr, q), v in p.halo_recv.items() if rr == r]
        for (q_dst, q_src) in pairs:
            for d, s in zip(q_dst.tolist(), q_src.tolist()):
                assert owner(d) == r and d not in seen
                seen[d] = s
    for (r, q), (d, s) in p.halo_recv.items():
        assert all(owner(x) == q for x in s.tolist())
    assert seen == dict(zip(dst.tolist(), src.tolist()))
    # boundary values: what a rank's tiles, seam and pole passes read is computed by it or
    # received once, from the rank that computes it
    for r, (a, b) in enumerate(p.blocks):
        need = set(bsrc[a * p.gall:b * p.gall][bsrc[a * p.gall:b * p.gall] >= 0].tolist())
        if r == 0:
            need |= set(ring.ravel().tolist()) | {nb - 2, nb - 1}
        got = {}
        for (rr, q), lst in p.bval_recv.items():
            if rr != r:
                continue
            for x in lst.tolist():
                assert x not in got and owner(blist[x]) == q != r
                got[x] = q
        assert {x for x in need if owner(blist[x]) != r} == set(got)
    v_b, v_h = p.bytes_per_step(kall=8, ntr=2)
    assert v_b > 0 and v_h > 0


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist
    from icoatmosbenchmark_v1_b200 import api, shard
    dist.init_process_group("gloo", rank=rank, world_size=2)
    g, rl, m, K = 4, 1, 2, 3
    p = shard.ShardPlan.build(g, rl, 2)
    dst, src = api.comm_plan(g, rl)
    nb, bsrc, blist, ring = api.boundary_tables(g, rl)
    npt = p.nrgn * p.gall + 12
    rng = np.random.default_rng(11)
    R = rng.standard_normal((m, K, npt))      # every point's value before the fill
    V = rng.standard_normal((nb, 5, K))       # every boundary index's values
    mine = np.zeros(npt, bool)
    mine[p.owned_points(rank)] = True
    is_dst = np.zeros(npt, bool)
    is_dst[dst] = True
    X = np.full((m, K, npt), np.nan)
    X[:, :, mine & ~is_dst] = R[:, :, mine & ~is_dst]
    comp = np.array([0 if b >= npt - 12 else next(r for r, (a, c) in enumerate(p.blocks) if a <= b // p.gall < c)
                     for b in blist])
    B = np.full(V.shape, np.nan)
    B[comp == rank] = V[comp == rank]

    def swap(recv_key, send_key, send_arr, shape):
        reqs, buf = [], None
        if send_key in send_arr:
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(send_arr[send_key])), dst=1 - rank))
        if recv_key is not None:
            buf = torch.empty(shape, dtype=torch.float64)
            reqs.append(dist.irecv(buf, src=1 - rank))
        for q in reqs:
            q.wait()
        return None if buf is None else buf.numpy()

    # (1) boundary values, then (2) the halo fill; keys are (receiver, sender)
    other = 1 - rank
    sends = {}
    if (other, rank) in p.bval_recv:
        sends[(other, rank)] = B[p.bval_recv[(other, rank)]]
    lst = p.bval_recv.get((rank, other))
    got = swap((rank, other) if lst is not None else None, (other, rank), sends,
               (0 if lst is None else lst.size, 5, K))
    if lst is not None:
        B[lst] = got
    sends = {}
    if (other, rank) in p.halo_recv:
        sends[(other, rank)] = X[:, :, p.halo_recv[(other, rank)][1]]
    pr = p.halo_recv.get((rank, other))
    got = swap((rank, other) if pr is not None else None, (other, rank), sends,
               (m, K, 0 if pr is None else pr[0].size))
    if pr is not None:
        X[:, :, pr[0]] = got
    ld, ls = p.halo_local[rank]
    X[:, :, ld] = X[:, :, ls]
    # what the rank reads after the fill equals the single-process fill
    ref = R.copy()
    ref[:, :, dst] = ref[:, :, src]
    a, b = p.blocks[rank]
    own_dst = dst[(dst < npt - 12) & (dst // p.gall >= a) & (dst // p.gall < b)] if rank else \
        dst[((dst < npt - 12) & (dst // p.gall >= a) & (dst // p.gall < b)) | (dst >= npt - 12)]
    ok_halo = bool(np.array_equal(X[:, :, own_dst], ref[:, :, own_dst]))
    need = bsrc[a * p.gall:b * p.gall]
    need = np.unique(need[need >= 0])
    if rank == 0:
        need = np.unique(np.concatenate([need, ring.ravel(), [nb - 2, nb - 1]]))
    ok_bval = bool(np.array_equal(B[need], V[need]))
    dist.destroy_process_group()
    Path(out, f"rank{rank}.json").write_text(json.dumps({"halo": ok_halo, "bval": ok_bval,
                                                        "nhalo": int(own_dst.size), "nneed": int(need.size)}))


def test_two_rank_exchange_gloo(tmp_path, built):
    import torch.multiprocessing as mp
    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    mp.start_processes(_exchange_worker, args=(_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in (0, 1):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d["halo"] and d["bval"] and d["nhalo"] > 0 and d["nneed"] > 0, d


@pytest.mark.parametrize("glevel,rlevel", [(4, 0), (4, 1), (5, 2)])
def test_boundary_tables(built, glevel, rlevel):
    """ica_boundary_tables, the tables the batched step reads: boundary indices of the region
    edge cells in order, then the two pole centres; a halo point takes its plan source's
    index; every pole ring slot has one; interior cells off the edge -1, unwritten halo -2."""
    from icoatmosbenchmark_v1_b200 import api
    nb, bsrc, blist, ring = api.boundary_tables(glevel, rlevel)
    g1 = 2 ** (glevel - rlevel) + 2
    gall, L = g1 * g1, 10 * 4 ** rlevel
    npt = L * gall
    ij = np.arange(gall)
    i, j = ij % g1 + 1, ij // g1 + 1
    inner = (i >= 2) & (i <= g1 - 1) & (j >= 2) & (j <= g1 - 1)
    edge = inner & ((i == 2) | (i == g1 - 1) | (j == 2) | (j == g1 - 1))
    cells = (np.arange(L)[:, None] * gall + ij[edge][None, :]).ravel()
    np.testing.assert_array_equal(blist, np.concatenate([cells, [npt, npt + 6]]))
    np.testing.assert_array_equal(bsrc[cells], np.arange(cells.size))
    b2 = bsrc.reshape(L, gall)
    assert (b2[:, inner & ~edge] == -1).all()
    dst, src = api.comm_plan(glevel, rlevel)
    rd = dst < npt
    exp = np.where(src[rd] < npt, bsrc[np.minimum(src[rd], npt - 1)], cells.size + (src[rd] - npt) // 6)
    np.testing.assert_array_equal(bsrc[dst[rd]], exp)
    assert ((ring >= 0) & (ring < nb)).all()
    halo = np.ones(npt, bool)
    halo[(np.arange(L)[:, None] * gall + ij[inner][None, :]).ravel()] = False
    unwritten = halo.copy()
    unwritten[dst[rd]] = False
    assert (bsrc[unwritten] == -2).all()


class _FakeCtx:
    """Stands in for a sharded context on CPU: part 1 puts the rank's boundary values (those its
    own regions and, on rank 0, the pole centres compute) into its boundary buffer, part 2 the
    rank's own points of the next state, then the rank's own halo copies; the values come from a
    whole-grid reference, so after the runner's exchanges every rank must hold the reference's
    values wherever it reads."""

    def __init__(self, ref_state, ref_bval, blist, gall, nrgn, backend):
        self.ref, self.ref_b, self.blist, self.gall, self.nrgn, self.be = ref_state, ref_bval, blist, gall, nrgn, backend

    def shard_set(self, l0, l1, poles, dst, src):
        self.l0, self.l1, self.poles = l0, l1, poles
        import torch
        self.local = (torch.as_tensor(np.asarray(dst, np.int64)), torch.as_tensor(np.asarray(src, np.int64)))

    def _own(self, pts):
        pts = np.asarray(pts)
        l = pts // self.gall
        return np.where(pts >= self.nrgn * self.gall, bool(self.poles), (l >= self.l0) & (l < self.l1))

    def advect_fast_part_dev(self, part, dt, a, b, f):
        import torch
        if part == 1:
            own = torch.as_tensor(self._own(self.blist))
            self.be.bbuf[:, :, own] = self.ref_b[:, :, own]
            return
        npt = self.nrgn * self.gall + 12
        own = torch.as_tensor(self._own(np.arange(npt)))
        for k, kp in (("rhog", "rhog_pl"), ("rhogq", "rhogq_pl")):
            v, vp = (b[k].unsqueeze(0), b[kp].unsqueeze(0)) if k == "rhog" else (b[k], b[kp])
            rv, rvp = (self.ref[k].unsqueeze(0), self.ref[kp].unsqueeze(0)) if k == "rhog" else (self.ref[k], self.ref[kp])
            fl = self.be._flat(v, vp)
            fl[:, :, own] = self.be._flat(rv, rvp)[:, :, own]
            fl[:, :, self.local[0]] = fl[:, :, self.local[1]]
            m, L, K, G = v.shape
            v.copy_(fl[:, :, :L * G].reshape(m, K, L, G).permute(0, 2, 1, 3))
            vp.copy_(fl[:, :, L * G:].reshape(m, K, 2, 6).permute(0, 2, 1, 3))


def _runner_worker(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist
    from icoatmosbenchmark_v1_b200 import api, shard
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        g, rl, K, T = 4, 0, 5, 3
        plan = shard.ShardPlan.build(g, rl, 2)
        L, gall = plan.nrgn, plan.gall
        nb, bsrc, blist, ring = api.boundary_tables(g, rl)
        gen = torch.Generator().manual_seed(5)
        # the whole-grid reference: any values, halos filled by the composed plan
        ref = {"rhog": torch.rand((L, K, gall), generator=gen, dtype=torch.float64),
               "rhog_pl": torch.rand((2, K, 6), generator=gen, dtype=torch.float64),
               "rhogq": torch.rand((T, L, K, gall), generator=gen, dtype=torch.float64),
               "rhogq_pl": torch.rand((T, 2, K, 6), generator=gen, dtype=torch.float64)}
        dst, src = api.comm_plan(g, rl)
        be0 = shard.TorchBackend()
        for k, kp in (("rhog", "rhog_pl"), ("rhogq", "rhogq_pl")):
            v, vp = (ref[k].unsqueeze(0), ref[kp].unsqueeze(0)) if k == "rhog" else (ref[k], ref[kp])
            fl = be0._flat(v, vp)
            fl[:, :, torch.as_tensor(dst.astype(np.int64))] = fl[:, :, torch.as_tensor(src.astype(np.int64))]
            m = v.shape[0]
            v.copy_(fl[:, :, :L * gall].reshape(m, K, L, gall).permute(0, 2, 1, 3))
            vp.copy_(fl[:, :, L * gall:].reshape(m, K, 2, 6).permute(0, 2, 1, 3))
        ref_b = torch.rand((T, K, nb, 5), generator=gen, dtype=torch.float64)
        nan = lambda t: torch.full_like(t, float("nan"))  # noqa: E731
        state = {k: nan(v) for k, v in ref.items()}
        fields = {k: torch.zeros((L, K, gall) if not k.endswith("_pl") else (2, K, 6)) for k in api.FIELD_KEYS}
        be = shard.TorchBackend(torch.full((T, K, nb, 5), float("nan"), dtype=torch.float64))
        ctx = _FakeCtx(ref, ref_b, blist, gall, L, be)
        run = shard.ShardedRunner(ctx, plan, rank, state, fields, 1.0, backend=be)
        run.step()
        S = run.state
        # every point this rank owns (its regions' interior and halo, and on rank 0 the poles)
        own = plan.owned_points(rank)
        ok_state = all(torch.equal(be0._flat(*((S[k].unsqueeze(0), S[kp].unsqueeze(0)) if k == "rhog"
                                                 else (S[k], S[kp])))[:, :, own],
                                   be0._flat(*((ref[k].unsqueeze(0), ref[kp].unsqueeze(0)) if k == "rhog"
                                               else (ref[k], ref[kp])))[:, :, own])
                       for k, kp in (("rhog", "rhog_pl"), ("rhogq", "rhogq_pl")))
        # every boundary value it reads
        a0, a1 = plan.blocks[rank]
        need = bsrc[a0 * gall:a1 * gall]
        need = need[need >= 0]
        if rank == 0:
            need = np.concatenate([need, ring.ravel(), nb - 2 + np.arange(2)])
        need = torch.as_tensor(np.unique(need).astype(np.int64))
        ok_bval = torch.equal(be.bbuf[:, :, need], ref_b[:, :, need])
        Path(out, f"r{rank}.json").write_text(json.dumps({"state": bool(ok_state), "bval": bool(ok_bval),
                                                          "backend": dist.get_backend()}))
    finally:
        dist.destroy_process_group()


def test_sharded_runner_step_two_ranks_gloo(tmp_path, built):
    """ShardedRunner.step on two gloo ranks (the CPU stand-in of NCCL): its boundary-value and
    halo exchanges (p2p_exchange along the plan's lists, torch pack / unpack) leave each rank
    with the whole-grid values at every point it owns and every boundary value it reads, bit
    for bit."""
    import torch.multiprocessing as mp
    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    mp.start_processes(_runner_worker, args=(_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in (0, 1):
        d = json.loads((tmp_path / f"r{r}.json").read_text())
        assert d == {"state": True, "bval": True, "backend": "gloo"}, (r, d)
