"""GPU tests of batches of uneven grid instances advanced by the same launches
(ica_batch_*): identical to advancing each instance alone, identical when replayed
from the captured CUDA graph, within 1e-5 of the FP64 oracle (FP32 variant) and equal
to it (FP64 variant, the plain path), and conserving mass."""
import numpy as np
import pytest

from cases import case, rel_err

pytestmark = pytest.mark.gpu
PAIRS = [((4, 0, 10, 3), (3, 0, 6, 2)), ((5, 0, 12, 4), (4, 1, 10, 2))]


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


@pytest.mark.parametrize("pair", PAIRS)
def test_batch_equals_each_instance_alone_and_graph_replay(pair):
    import torch
    from icoatmosbenchmark_v1_b200 import api
    cs = [case(*p) for p in pair]
    ctxs = [_ctx(c["grid"]) for c in cs]
    try:
        singles = []
        for c, ctx in zip(cs, ctxs):
            r = ctx.fast_runner(c["grid"], _dev(c["state"]), _dev(c["fields"]), c["dt"], autotune=False)
            ctx.fast_set_shape(0)
            for _ in range(3):
                r.step()
            torch.cuda.synchronize()
            singles.append({k: v.cpu().numpy() for k, v in r.state.items()})
        br = api.BatchRunner(ctxs, [_dev(c["state"]) for c in cs], [_dev(c["fields"]) for c in cs],
                             [c["dt"] for c in cs], shape=0)
        br.step()  # uncaptured: sets up every buffer
        n0 = sum(c.launch_count for c in ctxs)
        br.step()
        per_step = sum(c.launch_count for c in ctxs) - n0
        br.use_graph()
        n0 = sum(c.launch_count for c in ctxs)
        br.step()
        torch.cuda.synchronize()
        # a replay counts the kernels its graph launches, as an uncaptured step does
        assert per_step > 0 and sum(c.launch_count for c in ctxs) - n0 == per_step
        for got, ref in zip(br.states, singles):
            for k in ref:
                np.testing.assert_array_equal(got[k].cpu().numpy(), ref[k], err_msg=k)
        br.close()
    finally:
        for ctx in ctxs:
            ctx.close()


def test_batch_fp32_and_fp64_against_oracle(O):
    """Uneven pair, 2 steps: the batched FP32 variant within 1e-5 of the FP64 oracle; the FP64
    variant (plain path, instance by instance) equal to it bit for bit."""
    import torch
    from icoatmosbenchmark_v1_b200 import api
    cs = [case(*p) for p in PAIRS[1]]
    ctxs = [_ctx(c["grid"]) for c in cs]
    try:
        refs = []
        for c in cs:
            S = {k: v.copy() for k, v in c["state"].items()}
            for _ in range(2):
                O.step(c["dims"], c["grid"].have_sgp, c["topo"], c["dt"], S, c["fields"], c["grid"].arrays,
                       nthreads=8)
            refs.append(S)
        br = api.BatchRunner(ctxs, [_dev(c["state"]) for c in cs], [_dev(c["fields"]) for c in cs],
                             [c["dt"] for c in cs], shape=3)
        for _ in range(2):
            br.step()
        torch.cuda.synchronize()
        for got, ref in zip(br.states, refs):
            for k in ref:
                assert rel_err(got[k].cpu().numpy(), ref[k]) <= 1e-5, k
        br.close()
        for c, ctx, ref in zip(cs, ctxs, refs):
            G = {k: v.copy() for k, v in c["state"].items()}
            f = c["fields"]
            for _ in range(2):
                ctx.advect_step(c["dt"], G["rhog"], G["rhog_pl"], G["rhogq"], G["rhogq_pl"], f["rhogvx"],
                                f["rhogvx_pl"], f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"],
                                f["rhogw"], f["rhogw_pl"])
            for k in ref:
                np.testing.assert_array_equal(G[k], ref[k], err_msg=k)
    finally:
        for ctx in ctxs:
            ctx.close()


def test_batch_mass_conservation_uneven():
    """gl6 kall 42 (4 tracers) with gl5 kall 12 (2 tracers), 6 graph-replayed steps: relative
    mass drift of every tracer of both instances <= 1e-12."""
    import torch
    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    grids = [Grid(6, 0, 42), Grid(5, 0, 12)]
    ntrs = [4, 2]
    fs = [{k: v.cuda() for k, v in F.make_fields(g).items()} for g in grids]
    sts = [{k: v.cuda() for k, v in F.make_state(g, n, "mixed").items()} for g, n in zip(grids, ntrs)]
    ctxs = [_ctx(g) for g in grids]

    def mass(g, S):
        m = torch.as_tensor(g.interior_mask(), device="cuda")
        kk = slice(g.kmin - 1, g.kmax)
        area = torch.as_tensor(g.arrays["GMTR_p"][0], device="cuda")
        dz = torch.as_tensor(g.arrays["dz"], device="cuda")
        apl = torch.as_tensor(g.arrays["GMTR_p_pl"][0][:, 0], device="cuda")
        a = (S["rhogq"][:, :, kk] * (area * m)[None, :, None] * dz[kk][None, None, :, None]).sum((1, 2, 3))
        return a + (S["rhogq_pl"][:, :, kk, 0] * apl[None, :, None] * dz[kk][None, None]).sum((1, 2))

    try:
        m0 = [mass(g, s) for g, s in zip(grids, sts)]
        br = api.BatchRunner(ctxs, sts, fs, [default_dt(g.glevel) for g in grids], shape=0)
        br.step()
        br.use_graph()
        for _ in range(5):
            br.step()
        torch.cuda.synchronize()
        for g, S, m in zip(grids, br.states, m0):
            drift = ((mass(g, S) - m).abs() / m.abs()).max().item()
            assert drift <= 1e-12, drift
        br.close()
    finally:
        for ctx in ctxs:
            ctx.close()


def test_fp64_variant_batch_against_oracle(O):
    """The FP64 variant of the batched step (FP64 fields, faces and limiters in the same
    persistent launches, replayed from the captured CUDA graph): uneven pair, 3 steps, within
    1e-11 of the FP64 oracle (the operation order differs from the plain step's)."""
    import torch
    from icoatmosbenchmark_v1_b200 import api
    cs = [case(*p) for p in PAIRS[1]]
    ctxs = [_ctx(c["grid"]) for c in cs]
    try:
        refs = []
        for c in cs:
            S = {k: v.copy() for k, v in c["state"].items()}
            for _ in range(3):
                O.step(c["dims"], c["grid"].have_sgp, c["topo"], c["dt"], S, c["fields"], c["grid"].arrays,
                       nthreads=8)
            refs.append(S)
        br = api.BatchRunner(ctxs, [_dev(c["state"]) for c in cs], [_dev(c["fields"]) for c in cs],
                             [c["dt"] for c in cs], shape=3, f64=True)
        br.step()
        br.use_graph()
        br.step()
        br.step()
        torch.cuda.synchronize()
        for got, ref in zip(br.states, refs):
            for k in ref:
                assert rel_err(got[k].cpu().numpy(), ref[k]) <= 1e-11, k
        br.close()
    finally:
        for ctx in ctxs:
            ctx.close()


@pytest.mark.parametrize("glevel,rlevel,kall,ntr", [(5, 0, 42, 3), (4, 1, 10, 2)])
def test_fp64_variant_single_grid_against_plain_step(glevel, rlevel, kall, ntr):
    """ica_advect_fast64_dev against the plain FP64 step on the same inputs, 3 steps: 1e-11."""
    import torch
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    ctx = _ctx(g)
    try:
        P = _dev(c["state"])
        A, B = _dev(c["state"]), {k: torch.empty_like(v) for k, v in _dev(c["state"]).items()}
        fd = _dev(f)
        for _ in range(3):
            ctx.advect_step(c["dt"], P["rhog"], P["rhog_pl"], P["rhogq"], P["rhogq_pl"], fd["rhogvx"], fd["rhogvx_pl"],
                            fd["rhogvy"], fd["rhogvy_pl"], fd["rhogvz"], fd["rhogvz_pl"], fd["rhogw"], fd["rhogw_pl"])
            ctx.advect_fast64_dev(c["dt"], A, B, fd)
            A, B = B, A
        torch.cuda.synchronize()
        for k in P:
            assert rel_err(A[k].cpu().numpy(), P[k].cpu().numpy()) <= 1e-11, k
    finally:
        ctx.close()


def test_uneven_batch_full_size_against_plain_fp64():
    """The uneven batch at its full size (glevel 7 / kall 96 / 40 tracers and glevel 6 / kall 42 /
    12 tracers, half the tracers spherical-harmonic fields and half slotted cylinders), one
    launch per stage over both instances, replayed from the CUDA graph: after 2 steps the FP32
    variant is within 1e-5 of the plain FP64 step (bit-exact to the oracle at smaller sizes)
    and the FP64 variant within 1e-11, and both conserve mass to 1e-12."""
    import torch
    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid, default_dt
    import bench
    dev = torch.device("cuda")
    grids = [Grid(gl, 0, K) for gl, K, _ in bench.UNEVEN]
    ctxs, fs, sts, dts = [], [], [], []
    for g, (gl, K, T) in zip(grids, bench.UNEVEN):
        f = F.make_fields(g, device=dev)
        sts.append(F.make_state(g, T, "mixed", device=dev, fields=f))
        fs.append(f)
        ctx = api.IcoAdv(gl, 0, K - 2)
        ctx.set_grid(g)
        ctxs.append(ctx)
        dts.append(default_dt(gl))
    try:
        refs = []
        for ctx, st, f, dt in zip(ctxs, sts, fs, dts):
            S = {k: v.clone() for k, v in st.items()}
            for _ in range(2):
                ctx.advect_step(dt, S["rhog"], S["rhog_pl"], S["rhogq"], S["rhogq_pl"], f["rhogvx"], f["rhogvx_pl"],
                                f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], f["rhogw"], f["rhogw_pl"])
            refs.append(S)
        for f64, tol in ((False, 1e-5), (True, 1e-11)):
            br = api.BatchRunner(ctxs, [{k: v.clone() for k, v in st.items()} for st in sts], fs, dts, shape=3,
                                 f64=f64)
            m0 = [bench.tracer_mass(g, S) for g, S in zip(grids, br.states)]
            br.step()  # uncaptured: sets up every buffer
            br.use_graph()
            br.step()
            torch.cuda.synchronize()
            for got, ref in zip(br.states, refs):
                for k in ("rhog", "rhogq"):
                    e = float(((got[k] - ref[k]).abs().max() / ref[k].abs().max()).item())
                    assert e <= tol, (f64, k, e)
            m1 = [bench.tracer_mass(g, S) for g, S in zip(grids, br.states)]
            for a, b in zip(m0, m1):
                assert float(((b - a).abs() / a.abs()).max().item()) <= 1e-12
            br.close()
            del br
            torch.cuda.empty_cache()
    finally:
        for ctx in ctxs:
            ctx.close()
