"""Region sharding of the batched step on the device (ica_shard_set, ica_advect_fast_part_dev,
ica_shard_*_pack/unpack), with the ranks emulated in one process on one GPU: each rank has its
own context and state buffers, computes its block of regions, and the exchanges copy packed
buffers between the ranks (no kernel waits for another rank's).  The sharded steps equal the
whole-grid batched step bit for bit at every point each rank owns: the same kernels compute
every value from bit-identical inputs."""
import numpy as np
import pytest

from cases import case

pytestmark = pytest.mark.gpu


def _dev(d):
    import torch
    return {k: torch.as_tensor(v, device="cuda").contiguous() for k, v in d.items()}


def _flat(S):
    import torch
    from icoatmosbenchmark_v1_b200.shard import TorchBackend
    return torch.cat([TorchBackend._flat(S["rhog"].unsqueeze(0), S["rhog_pl"].unsqueeze(0)),
                      TorchBackend._flat(S["rhogq"], S["rhogq_pl"])], 0)


@pytest.mark.parametrize("glevel,rlevel,kall,ntr,nranks,nsteps", [(5, 0, 10, 5, 2, 2), (4, 1, 8, 3, 3, 2),
                                                                   (4, 0, 6, 2, 10, 1)])
def test_emulated_ranks_equal_whole_grid(built, cuda, glevel, rlevel, kall, ntr, nranks, nsteps):
    import torch
    from icoatmosbenchmark_v1_b200 import api, shard
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    ctx = api.IcoAdv(glevel, rlevel, kall - 2)
    ctx.set_grid(g)
    ctxs = []
    try:
        r = ctx.fast_runner(g, _dev(c["state"]), _dev(f), c["dt"], autotune=False)
        for _ in range(nsteps):
            r.step()
        ref = _flat(r.state)
        plan = shard.ShardPlan.build(glevel, rlevel, nranks)
        runners = []
        for q in range(nranks):
            cq = api.IcoAdv(glevel, rlevel, kall - 2)
            cq.set_grid(g)
            ctxs.append(cq)
            runners.append(shard.ShardedRunner(cq, plan, q, _dev(c["state"]), _dev(f), c["dt"]))
        for _ in range(nsteps):
            shard.emulated_step(runners)
        torch.cuda.synchronize()
        for q, run in enumerate(runners):
            own = torch.as_tensor(plan.owned_points(q), device="cuda")
            got = _flat(run.state)[:, :, own]
            assert torch.equal(got, ref[:, :, own]), q
            assert ctxs[q].fast_status() == 0
    finally:
        ctx.close()
        for cq in ctxs:
            cq.close()


def test_pack_unpack_kernels_equal_torch_indexing(built, cuda):
    """The library's pack / unpack kernels against torch index operations on the same arrays."""
    import torch
    from icoatmosbenchmark_v1_b200 import api, shard
    g, rl, K, T = 4, 0, 6, 3
    ctx = api.IcoAdv(g, rl, K - 2)
    try:
        L, gall = ctx.sizes.lall, ctx.sizes.gall
        gen = torch.Generator(device="cuda").manual_seed(1)
        var = torch.rand((T, L, K, gall), generator=gen, dtype=torch.float64, device="cuda")
        var_pl = torch.rand((T, 2, K, 6), generator=gen, dtype=torch.float64, device="cuda")
        pts = torch.as_tensor(np.random.default_rng(2).choice(L * gall + 12, 500, replace=False).astype(np.int32),
                              device="cuda")
        lib_b, tb = shard.LibraryBackend(ctx), shard.TorchBackend()
        buf = lib_b.pack_points(pts, var, var_pl)
        assert torch.equal(buf, tb.pack_points(pts, var, var_pl))
        v2, vp2 = torch.zeros_like(var), torch.zeros_like(var_pl)
        lib_b.unpack_points(pts, v2, vp2, buf)
        v3, vp3 = torch.zeros_like(var), torch.zeros_like(var_pl)
        tb.unpack_points(pts, v3, vp3, buf)
        torch.cuda.synchronize()
        assert torch.equal(v2, v3) and torch.equal(vp2, vp3)
        # boundary values: through the context's boundary buffer
        nb = api.boundary_tables(g, rl)[0]
        bidx = torch.as_tensor(np.arange(0, nb, 7, dtype=np.int32), device="cuda")
        src = torch.rand((T, K, bidx.numel(), 5), generator=gen, dtype=torch.float64, device="cuda")
        lib_b.unpack_bval(T, K, bidx, src)
        back = lib_b.pack_bval(T, K, bidx)
        torch.cuda.synchronize()
        assert torch.equal(back, src)
    finally:
        ctx.close()
