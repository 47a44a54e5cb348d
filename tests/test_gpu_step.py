"""GPU parity of the composed step (plain FP64 per-tracer path) against the
oracle's composition, plus the properties the step must keep at sizes the
oracle does not reach quickly."""
import numpy as np
import pytest

from cases import case, interior, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


def _ctx(grid):
    from icoatmosbenchmark_v1_b200 import api
    ctx = api.IcoAdv(grid.glevel, grid.rlevel, grid.kall - 2)
    ctx.set_grid(grid)
    return ctx


@pytest.mark.parametrize("glevel,rlevel,kall,ntr,nsteps",
                         [(5, 0, 42, 8, 10), (5, 0, 42, 2, 3), (4, 1, 10, 3, 2), (3, 0, 6, 1, 4)])
def test_plain_step_bit_exact(O, glevel, rlevel, kall, ntr, nsteps):
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    S = {k: v.copy() for k, v in c["state"].items()}
    G = {k: v.copy() for k, v in c["state"].items()}
    ctx = _ctx(g)
    try:
        for _ in range(nsteps):
            O.step(c["dims"], g.have_sgp, c["topo"], c["dt"], S, f, g.arrays, nthreads=8)
            ctx.advect_step(c["dt"], G["rhog"], G["rhog_pl"], G["rhogq"], G["rhogq_pl"], f["rhogvx"],
                            f["rhogvx_pl"], f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"],
                            f["rhogw_pl"])
        for k in ("rhog", "rhog_pl", "rhogq", "rhogq_pl"):
            assert rel_err(G[k], S[k]) <= 1e-12, k
            np.testing.assert_array_equal(G[k], S[k], err_msg=k)
    finally:
        ctx.close()


def test_plain_step_device_api_matches_host_api(O):
    import torch
    c = case(4, 0, 8, 2)
    g, f = c["grid"], c["fields"]
    ctx = _ctx(g)
    try:
        H = {k: v.copy() for k, v in c["state"].items()}
        D = {k: torch.as_tensor(v, device="cuda").contiguous() for k, v in c["state"].items()}
        fd = {k: torch.as_tensor(v, device="cuda").contiguous() for k, v in f.items()}
        ctx.advect_step(c["dt"], H["rhog"], H["rhog_pl"], H["rhogq"], H["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
        ctx.advect_step(c["dt"], D["rhog"], D["rhog_pl"], D["rhogq"], D["rhogq_pl"], fd["rhogvx"], fd["rhogvx_pl"],
                        fd["rhogvy"], fd["rhogvy_pl"], fd["rhogvz"], fd["rhogvz_pl"], fd["rhogw"], fd["rhogw_pl"])
        torch.cuda.synchronize()
        for k in H:
            np.testing.assert_array_equal(D[k].cpu().numpy(), H[k])
    finally:
        ctx.close()


def test_plain_step_conservation_constancy_monotonicity_gl6():
    """gl6, kall 42, 4 tracers (3 fields + a constant), 6 steps: mass drift <= 1e-12, a constant
    mixing ratio stays constant, bounded tracers stay in [0,1]."""
    import torch
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    g = Grid(6, 0, 42)
    f = {k: v.cuda() for k, v in F.make_fields(g).items()}
    st = {k: v.cuda() for k, v in F.make_state(g, 3, "mixed").items()}
    st["rhogq"] = torch.cat([st["rhogq"], 0.7 * st["rhog"][None]]).contiguous()
    st["rhogq_pl"] = torch.cat([st["rhogq_pl"], 0.7 * st["rhog_pl"][None]]).contiguous()
    ctx = _ctx(g)
    m = torch.as_tensor(g.interior_mask(), device="cuda")
    kk = slice(g.kmin - 1, g.kmax)
    area = torch.as_tensor(g.arrays["GMTR_p"][0], device="cuda")
    dz = torch.as_tensor(g.arrays["dz"], device="cuda")
    apl = torch.as_tensor(g.arrays["GMTR_p_pl"][0][:, 0], device="cuda")

    def mass(S):
        a = (S["rhogq"][:, :, kk] * (area * m)[None, :, None] * dz[kk][None, None, :, None]).sum((1, 2, 3))
        return a + (S["rhogq_pl"][:, :, kk, 0] * apl[None, :, None] * dz[kk][None, None]).sum((1, 2))

    try:
        m0 = mass(st)
        for _ in range(6):
            ctx.advect_step(default_dt(6), st["rhog"], st["rhog_pl"], st["rhogq"], st["rhogq_pl"], f["rhogvx"],
                            f["rhogvx_pl"], f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"],
                            f["rhogw_pl"])
        torch.cuda.synchronize()
        drift = ((mass(st) - m0).abs() / m0.abs()).max().item()
        assert drift <= 1e-12, drift
        q = (st["rhogq"] / st["rhog"][None])[:, :, kk]
        qi = q.permute(0, 2, 1, 3)[:, :, m]
        assert qi[:3].min().item() >= -1e-12 and qi[:3].max().item() <= 1 + 1e-12
        assert (qi[3] - 0.7).abs().max().item() < 1e-12
    finally:
        ctx.close()
