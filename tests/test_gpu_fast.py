"""GPU tests of the fused batched path (FP32 flux/limiter, FP64 mass update):
error against the FP64 oracle's composed step, conservation, monotonicity,
constancy, every tile shape, and host vs device entry points."""
import numpy as np
import pytest

from cases import case, rel_err

pytestmark = pytest.mark.gpu
FP32_TOL = 1e-5


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


def _dev(d):
    import torch
    return {k: torch.as_tensor(v, device="cuda").contiguous() for k, v in d.items()}


def _ctx(grid):
    from icoatmosbenchmark_v1_b200 import api
    ctx = api.IcoAdv(grid.glevel, grid.rlevel, grid.kall - 2)
    ctx.set_grid(grid)
    return ctx


# kall 4, 5, 7 and 8 with the others: each way the column kernel's level loop can end (its three
# window slots for the top level, the remainder levels, no full three-level group at all), with
# full and partial last tracer groups (5 and 9 tracers: groups of 4 then 1)
@pytest.mark.parametrize("glevel,rlevel,kall,ntr,nsteps", [(5, 0, 42, 5, 3), (4, 1, 10, 3, 2), (6, 0, 12, 2, 2),
                                                           (3, 0, 6, 1, 2), (4, 0, 4, 5, 2), (4, 0, 5, 9, 2),
                                                           (4, 0, 7, 4, 2), (4, 0, 8, 6, 2)])
def test_fast_matches_fp64_oracle(O, glevel, rlevel, kall, ntr, nsteps):
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    S = {k: v.copy() for k, v in c["state"].items()}
    ctx = _ctx(g)
    try:
        r = ctx.fast_runner(g, _dev(c["state"]), _dev(f), c["dt"], autotune=False)
        for _ in range(nsteps):
            O.step(c["dims"], g.have_sgp, c["topo"], c["dt"], S, f, g.arrays, nthreads=8)
            r.step()
        got = {k: v.cpu().numpy() for k, v in r.state.items()}
        assert ctx.fast_status() == 0  # every wait of the tile kernel for its TMA copies ended in time
        for k in ("rhog", "rhog_pl", "rhogq", "rhogq_pl"):
            e = rel_err(got[k], S[k])
            assert e <= FP32_TOL, (k, e)
    finally:
        ctx.close()


@pytest.mark.parametrize("ntr", [9, 8])  # odd and even counts of 4-tracer batches (a CTA's levels chain their copies)
def test_fast_every_tile_shape(O, ntr):
    import torch
    c = case(5, 0, 12, ntr)
    g, f = c["grid"], c["fields"]
    S = {k: v.copy() for k, v in c["state"].items()}
    O.step(c["dims"], g.have_sgp, c["topo"], c["dt"], S, f, g.arrays, nthreads=8)
    ctx = _ctx(g)
    try:
        outs = []
        for s in range(len(ctx.fast_shapes())):
            r = ctx.fast_runner(g, _dev(c["state"]), _dev(f), c["dt"], autotune=False)
            ctx.fast_set_shape(s)
            r.step()
            torch.cuda.synchronize()
            got = r.state["rhogq"].cpu().numpy()
            assert rel_err(got, S["rhogq"]) <= FP32_TOL, s
            outs.append(got)
        assert ctx.fast_status() == 0
        for o in outs[1:]:  # the tile shape does not change any result
            np.testing.assert_array_equal(o, outs[0])
    finally:
        ctx.close()


@pytest.mark.parametrize("ntr,chunk,pinned", [(3, 0, False), (9, 0, False), (9, 0, True), (9, 2, True),
                                               (5, 1, False)])
def test_fast_host_entry_equals_device_entry(ntr, chunk, pinned):
    """The host-pointer step moves the state in chunks of tracers, overlapping the copies with
    the step (9 tracers by size at this grid: chunks 4, 4, 1, both staging slots reused); its
    result is the device step's, bit for bit, whatever the chunk, from pageable or pinned
    host memory."""
    import torch
    c = case(4, 0, 8, ntr)
    g, f = c["grid"], c["fields"]
    ctx = _ctx(g)
    try:
        ctx.fast_set_host_chunk(chunk)
        r = ctx.fast_runner(g, _dev(c["state"]), _dev(f), c["dt"], autotune=False)
        r.step()
        torch.cuda.synchronize()
        if pinned:
            H = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in c["state"].items()}
        else:
            H = {k: v.copy() for k, v in c["state"].items()}
        f32 = {k: np.ascontiguousarray(f[k], np.float32) for k in ("rhogvx", "rhogvx_pl", "rhogvy", "rhogvy_pl",
                                                                  "rhogvz", "rhogvz_pl", "rhogw", "rhogw_pl")}
        ctx.advect_fast_host(c["dt"], H["rhog"], H["rhog_pl"], H["rhogq"], H["rhogq_pl"], **f32)
        for k in H:
            np.testing.assert_array_equal(H[k], r.state[k].cpu().numpy())
    finally:
        ctx.close()


def test_fast_conservation_monotonicity_constancy_gl6():
    """gl6 kall 42, 4 mixed tracers + a constant, 8 steps: relative mass drift <= 1e-12 (FP64
    update, seam faces in FP64), bounded tracers stay in [0,1] to 1e-6, constant stays constant."""
    import torch
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    g = Grid(6, 0, 42)
    f = {k: v.cuda() for k, v in F.make_fields(g).items()}
    st = {k: v.cuda() for k, v in F.make_state(g, 4, "mixed").items()}
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
        r = ctx.fast_runner(g, st, f, default_dt(6), autotune=False)
        for _ in range(8):
            r.step()
        torch.cuda.synchronize()
        S = r.state
        drift = ((mass(S) - m0).abs() / m0.abs()).max().item()
        assert drift <= 1e-12, drift
        q = (S["rhogq"] / S["rhog"][None])[:, :, kk]
        qi = q.permute(0, 2, 1, 3)[:, :, m]
        assert qi[:4].min().item() >= -1e-6 and qi[:4].max().item() <= 1 + 1e-6
        assert (qi[4] - 0.7).abs().max().item() < 1e-6
    finally:
        ctx.close()


def test_fast_full_size_gl8_k96_32_tracers():
    """The headline workload at full size (glevel 8, kall 96, 31 mixed tracers and a constant):
    the first batched step against the plain FP64 step (bit-exact to the oracle at the smaller
    sizes) within 1e-5 relative, then 3 more steps: relative mass drift <= 1e-12, bounded tracers
    in [0, 1] to 1e-6, the constant tracer constant to 1e-6."""
    import torch
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    g = Grid(8, 0, 96)
    dt = default_dt(8)
    f = F.make_fields(g, device="cuda")
    st = F.make_state(g, 31, "mixed", device="cuda", fields=f)
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
        ref = {k: v.clone() for k, v in st.items()}
        ctx.advect_step(dt, ref["rhog"], ref["rhog_pl"], ref["rhogq"], ref["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
        fields = {k: v for k, v in f.items() if k not in ("rhog", "rhog_pl")}
        r = ctx.fast_runner(g, st, fields, dt, autotune=False)
        r.step()
        torch.cuda.synchronize()
        for k in ("rhog", "rhogq"):
            e = ((r.state[k] - ref[k]).abs().max() / ref[k].abs().max()).item()
            assert e <= FP32_TOL, (k, e)
        del ref
        for _ in range(3):
            r.step()
        torch.cuda.synchronize()
        S = r.state
        drift = ((mass(S) - m0).abs() / m0.abs()).max().item()
        assert drift <= 1e-12, drift
        q = (S["rhogq"] / S["rhog"][None])[:, :, kk]
        lo = hi = None
        for t in range(31):  # one tracer at a time: the interior gather of all 31 would be 15 GB
            qi = q[t].permute(1, 0, 2)[:, m]
            lo = qi.min().item() if lo is None else min(lo, qi.min().item())
            hi = qi.max().item() if hi is None else max(hi, qi.max().item())
        assert lo >= -1e-6 and hi <= 1 + 1e-6, (lo, hi)
        assert (q[31].permute(1, 0, 2)[:, m] - 0.7).abs().max().item() < 1e-6
    finally:
        ctx.close()
