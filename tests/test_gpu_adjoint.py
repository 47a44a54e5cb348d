"""GPU adjoint of the plain FP64 step through the C ABI (ica_advect_step_adjoint,
ica_adjoint_record / ica_adjoint_sweep).

Checked against the oracle's adjoint (the FP64 reference gradient) on the same
seeded inputs, against central finite differences of the GPU forward step away
from limiter kinks, and through a torch.autograd.Function wrapper (defined
here, in the test harness only) over a checkpointed multi-step run.

The tracer fields get seeded noise of 1e-3 relative.  The slotted cylinder's
flat regions are exact ties of every min / max / clamp (value = bound = 0 or
1), where the forward's branch is a subgradient that coordinate differences
cannot see; the noise breaks the ties."""
import numpy as np
import pytest

from cases import case

pytestmark = pytest.mark.gpu

STATE = ("rhog", "rhog_pl", "rhogq", "rhogq_pl")
WIND = ("rhogvx", "rhogvx_pl", "rhogvy", "rhogvy_pl", "rhogvz", "rhogvz_pl")


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


def _ctx(grid):
    from icoatmosbenchmark_v1_b200 import api
    ctx = api.IcoAdv(grid.glevel, grid.rlevel, grid.kall - 2)
    ctx.set_grid(grid)
    return ctx


def _noisy(state, seed=11, amp=1e-3):
    rng = np.random.default_rng(seed)
    S = {k: v.copy() for k, v in state.items()}
    S["rhogq"] = S["rhogq"] + amp * S["rhog"][None] * rng.random(S["rhogq"].shape)
    S["rhogq_pl"] = S["rhogq_pl"] + amp * S["rhog_pl"][None] * rng.random(S["rhogq_pl"].shape)
    return S


def _close(g, ref, rtol, name):
    scale = float(np.abs(ref).max())
    err = float(np.abs(g - ref).max())
    assert err <= rtol * max(scale, 1e-300), f"{name}: max |gpu - ref| {err:.3e} vs max |ref| {scale:.3e}"


@pytest.mark.parametrize("glevel,rlevel,kall,ntr", [(3, 0, 6, 2), (4, 1, 10, 2), (5, 0, 12, 3)])
def test_step_adjoint_matches_oracle(O, glevel, rlevel, kall, ntr):
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    S0 = _noisy(c["state"])
    rng = np.random.default_rng(5)
    w = {k: rng.standard_normal(v.shape) for k, v in S0.items()}
    ref = {k: v.copy() for k, v in w.items()}
    ref_w = {k: np.zeros_like(f[k]) for k in WIND}
    O.step_adjoint(c["dims"], g.have_sgp, c["topo"], c["dt"], S0, f, g.arrays, ref, ref_w)
    got = {k: v.copy() for k, v in w.items()}
    got_w = {k: np.zeros_like(f[k]) for k in WIND}
    ctx = _ctx(g)
    try:
        ctx.advect_step_adjoint(c["dt"], S0, f, got, got_w)
    finally:
        ctx.close()
    for k in STATE:
        _close(got[k], ref[k], 1e-11, k)
    for k in WIND:
        _close(got_w[k], ref_w[k], 1e-11, k)


def test_step_adjoint_device_matches_host():
    import torch
    c = case(4, 0, 8, 2)
    g, f = c["grid"], c["fields"]
    S0 = _noisy(c["state"])
    rng = np.random.default_rng(6)
    w = {k: rng.standard_normal(v.shape) for k, v in S0.items()}
    ctx = _ctx(g)
    try:
        H = {k: v.copy() for k, v in w.items()}
        Hw = {k: np.zeros_like(f[k]) for k in WIND}
        ctx.advect_step_adjoint(c["dt"], S0, f, H, Hw)
        dv = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
        D = {k: dv(v) for k, v in w.items()}
        Dw = {k: dv(np.zeros_like(f[k])) for k in WIND}
        ctx.advect_step_adjoint(c["dt"], {k: dv(v) for k, v in S0.items()}, {k: dv(v) for k, v in f.items()}, D,
                                Dw)
        torch.cuda.synchronize()
        for k in STATE:
            _close(D[k].cpu().numpy(), H[k], 1e-13, k)
        for k in WIND:
            _close(Dw[k].cpu().numpy(), Hw[k], 1e-13, k)
    finally:
        ctx.close()


def _run(ctx, dt, S, F, nsteps):
    for _ in range(nsteps):
        ctx.advect_step(dt, S["rhog"], S["rhog_pl"], S["rhogq"], S["rhogq_pl"], F["rhogvx"], F["rhogvx_pl"],
                        F["rhogvy"], F["rhogvy_pl"], F["rhogvz"], F["rhogvz_pl"], F["rhogw"], F["rhogw_pl"])
    return S


def _central(dJ, S0, F0, which, idx, h0, grad, rtol, floor):
    """Central difference fd of J at element idx of S0[which] or F0[which] with step h0, checked
    for limiter kinks near the point.  J is piecewise smooth (piecewise linear in the tracer), so
    a kink at distance d < h0 biases fd by up to half its slope jump.  From J at +-h0 and +-2 h0
    (J at the point itself is 0, as dJ is a difference from it): the second-order one-sided
    differences (-3 J(0) + 4 J(+h) - J(+2h)) / 2h and its mirror agree to O(h^2) on a smooth
    piece, and so do the central differences at h0 and 2 h0.  A kink with d < h0 moves one or
    the other by at least the bias it puts on fd, so requiring both to agree to tau = rtol / 2
    leaves fd within tau of the slope at the point.  ('kink', fd) when they do not agree;
    away from kinks ('ok', fd) if |grad - fd| <= rtol max(|fd|, floor), else ('bad', fd)."""
    J = {}
    for m in (1, -1, 2, -2):
        S = {k: v.clone() for k, v in S0.items()}
        F = dict(F0)
        if which in S:
            S[which][idx] += m * h0
        else:
            F[which] = F0[which].clone()
            F[which][idx] += m * h0
        J[m] = dJ(S, F)
    h = h0
    fd = (J[1] - J[-1]) / (2 * h)
    fd2 = (J[2] - J[-2]) / (4 * h)
    right = (4 * J[1] - J[2]) / (2 * h)
    left = (J[-2] - 4 * J[-1]) / (2 * h)
    scale = max(abs(fd), floor)
    tau = 0.5 * rtol
    if abs(right - left) > tau * scale or abs(fd - fd2) > tau * scale:
        return "kink", fd
    return ("ok" if abs(grad - fd) <= rtol * scale else "bad"), fd


def _pick_interior(rng, g, shape, kall):
    while True:
        idx = tuple(int(rng.integers(0, s)) for s in shape)
        p, G = idx[-1], g.gall_1d
        i, j = p % G + 1, p // G + 1
        if g.gmin <= i <= g.gmax and g.gmin <= j <= g.gmax and 1 <= idx[-2] <= kall - 2:
            return idx


@pytest.mark.parametrize("glevel,rlevel,kall,ntr,nsteps", [(4, 0, 10, 2, 2), (3, 1, 8, 1, 3)])
def test_step_adjoint_against_finite_differences(glevel, rlevel, kall, ntr, nsteps):
    """J = sum w * state after nsteps GPU steps; central differences with h = 1e-6 of the
    field's largest magnitude, the difference of J taken as sum w * (S+ - S-) so that J's own
    size does not cancel."""
    import torch
    c = case(glevel, rlevel, kall, ntr)
    g, f = c["grid"], c["fields"]
    dt = c["dt"]
    dv = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
    S0 = {k: dv(v) for k, v in _noisy(c["state"]).items()}
    F0 = {k: dv(v) for k, v in f.items()}
    rng = np.random.default_rng(12)
    w = {k: dv(rng.standard_normal(tuple(v.shape))) for k, v in S0.items()}
    ctx = _ctx(g)
    try:
        states = [{k: v.clone() for k, v in S0.items()}]
        for _ in range(nsteps):
            states.append(_run(ctx, dt, {k: v.clone() for k, v in states[-1].items()}, F0, 1))
        a = {k: v.clone() for k, v in w.items()}
        aw = {k: torch.zeros_like(F0[k]) for k in WIND}
        for s in range(nsteps - 1, -1, -1):
            ctx.advect_step_adjoint(dt, states[s], F0, a, aw)
        end0 = states[-1]

        def dJ(S, F):  # J(S, F) - J(S0, F0) without forming J
            E = _run(ctx, dt, {k: v.clone() for k, v in S.items()}, F, nsteps)
            return float(sum((w[k] * (E[k] - end0[k])).sum() for k in E))

        checked = 0
        for n in range(36):
            which = ["rhogq", "rhog", "rhogvx", "rhogvy", "rhogvz", "rhogq"][n % 6]
            arr = S0[which] if which in S0 else F0[which]
            idx = _pick_interior(rng, g, tuple(arr.shape), kall)
            grad = float((a[which] if which in a else aw[which])[idx])
            h = 1e-6 * max(1.0, float(arr.abs().max()))
            status, fd = _central(dJ, S0, F0, which, idx, h, grad, 1e-6, 1e-3)
            assert status != "bad", (which, idx, grad, fd)
            checked += status == "ok"
        assert checked >= 25
    finally:
        ctx.close()


def _objective_seed(g, S, kr=(10, 20)):
    """J = sum of squared final tracer q = rhogq / rhog over region 0, levels kr (1-based,
    inclusive), interior points; returns J and dJ/d(rhog, rhogq) as device tensors."""
    import torch
    G = g.gall_1d
    ij = np.arange(g.gall)
    i, j = ij % G + 1, ij // G + 1
    inner = torch.as_tensor((i >= g.gmin) & (i <= g.gmax) & (j >= g.gmin) & (j <= g.gmax), device="cuda")
    mask = torch.zeros_like(S["rhog"], dtype=torch.bool)
    mask[0, kr[0] - 1:kr[1], :] = inner
    q = S["rhogq"] / S["rhog"][None]
    J = float((q * q)[:, mask].sum())
    aq = torch.where(mask[None], 2 * q / S["rhog"][None], torch.zeros_like(q))
    ar = torch.where(mask, -(2 * q * q / S["rhog"][None]).sum(0), torch.zeros_like(S["rhog"]))
    return J, mask, {"rhog": ar.contiguous(), "rhog_pl": torch.zeros_like(S["rhog_pl"]), "rhogq": aq.contiguous(),
                     "rhogq_pl": torch.zeros_like(S["rhogq_pl"])}


def _sweep(ctx, dt, nsteps, every, S0, F0):
    import torch
    S = {k: v.clone() for k, v in S0.items()}
    ctx.adjoint_record(dt, nsteps, every, S, F0)
    J, mask, a = _objective_seed(ctx._grid, S)
    aw = {k: torch.zeros_like(F0[k]) for k in WIND}
    ctx.adjoint_sweep(F0, a, aw)
    torch.cuda.synchronize()
    return J, mask, S, a, aw


def _ctx_dev(g):
    ctx = _ctx(g)
    ctx._grid = g
    return ctx


def test_checkpointed_sweep_matches_oracle(O):
    """A 6-step run with a checkpoint every 2 steps against the oracle's step adjoints
    chained over the oracle's own forward states."""
    import torch
    c = case(4, 0, 24, 2)
    g, f = c["grid"], c["fields"]
    dt = c["dt"]
    S0h = _noisy(c["state"])
    dv = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
    ctx = _ctx_dev(g)
    try:
        J, mask, Send, a, aw = _sweep(ctx, dt, 6, 2, {k: dv(v) for k, v in S0h.items()},
                                      {k: dv(v) for k, v in f.items()})
        states = [{k: v.copy() for k, v in S0h.items()}]
        for _ in range(6):
            S = {k: v.copy() for k, v in states[-1].items()}
            O.step(c["dims"], g.have_sgp, c["topo"], dt, S, f, g.arrays, nthreads=8)
            states.append(S)
        for k in STATE:  # the recorded run is the oracle's run, bit for bit
            np.testing.assert_array_equal(Send[k].cpu().numpy(), states[-1][k], err_msg=k)
        _, _, seed = _objective_seed(g, {k: dv(v) for k, v in states[-1].items()})
        ref = {k: v.cpu().numpy().copy() for k, v in seed.items()}
        ref_w = {k: np.zeros_like(f[k]) for k in WIND}
        for s in range(5, -1, -1):
            O.step_adjoint(c["dims"], g.have_sgp, c["topo"], dt, states[s], f, g.arrays, ref, ref_w)
        for k in STATE:
            _close(a[k].cpu().numpy(), ref[k], 1e-11, k)
        for k in WIND:
            _close(aw[k].cpu().numpy(), ref_w[k], 1e-11, k)
    finally:
        ctx.close()


def test_sweep_glevel6_kall42_8_tracers_24_steps():
    """The adjoint workload of 8 tracers on glevel 6, kall 42 over 24 steps, checkpoint every 6:
    the checkpointed sweep equals the sweep that keeps every state (checkpoint every step),
    and its gradients with respect to the initial tracer and the horizontal wind pass central
    differences at 64 seeded points away from limiter kinks, h = 1e-6 of the field's largest
    magnitude (an h relative to a small element itself drowns the difference in the rounding
    noise of the 24-step forward run)."""
    import torch
    c = case(6, 0, 42, 8)
    g, f = c["grid"], c["fields"]
    dt = c["dt"]
    dv = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
    S0 = {k: dv(v) for k, v in _noisy(c["state"]).items()}
    F0 = {k: dv(v) for k, v in f.items()}
    ctx = _ctx_dev(g)
    try:
        J, mask, Send, a, aw = _sweep(ctx, dt, 24, 6, S0, F0)
        _, _, _, a1, aw1 = _sweep(ctx, dt, 24, 1, S0, F0)
        for k in STATE:
            _close(a[k].cpu().numpy(), a1[k].cpu().numpy(), 1e-12, k)
        for k in WIND:
            _close(aw[k].cpu().numpy(), aw1[k].cpu().numpy(), 1e-12, k)
        ctx.adjoint_release()
        qend = Send["rhogq"] / Send["rhog"][None]

        def dJ(S, F):  # J(S, F) - J(S0, F0), summed as differences
            E = _run(ctx, dt, {k: v.clone() for k, v in S.items()}, F, 24)
            qe = E["rhogq"] / E["rhog"][None]
            return float(((qe - qend) * (qe + qend))[:, mask].sum())

        rng = np.random.default_rng(2024)
        # candidates: region 0 and its levels, where the gradient is not negligible
        cand = {"rhogq": a["rhogq"].abs(), "rhogvx": aw["rhogvx"].abs(), "rhogvy": aw["rhogvy"].abs(),
                "rhogvz": aw["rhogvz"].abs()}
        checked, kinks, worst = 0, 0, 0.0
        for n in range(200):
            if checked >= 64:
                break
            which = ["rhogq", "rhogvx", "rhogq", "rhogvy", "rhogq", "rhogvz"][n % 6]
            mag = cand[which]
            big = torch.nonzero(mag > 1e-2 * float(mag.max()))
            idx = tuple(int(v) for v in big[int(rng.integers(0, big.shape[0]))])
            grad = float((a[which] if which in a else aw[which])[idx])
            arr = S0[which] if which in S0 else F0[which]
            h = 1e-6 * float(arr.abs().max())
            status, fd = _central(dJ, S0, F0, which, idx, h, grad, 1e-6, 0.0)
            if status == "kink":
                kinks += 1
                continue
            rel = abs(grad - fd) / abs(fd)
            worst = max(worst, rel)
            assert status == "ok", (which, idx, grad, fd, rel)
            checked += 1
        assert checked >= 64, (checked, kinks)
        print(f"\nFD check: {checked} points, {kinks} skipped at kinks, worst relative error {worst:.2e}, J={J:.6e}")
    finally:
        ctx.close()


def test_autograd_function_wrapper():
    """torch.autograd.Function over a checkpointed run (test harness only): the gradient
    torch builds from J through the wrapper equals the direct sweep."""
    import torch

    class Advect(torch.autograd.Function):
        @staticmethod
        def forward(fctx, ica, dt, nsteps, every, fields, rhog, rhog_pl, rhogq, rhogq_pl, vx, vx_pl, vy, vy_pl,
                    vz, vz_pl):
            S = {"rhog": rhog.clone(), "rhog_pl": rhog_pl.clone(), "rhogq": rhogq.clone(),
                 "rhogq_pl": rhogq_pl.clone()}
            F = dict(fields, rhogvx=vx, rhogvx_pl=vx_pl, rhogvy=vy, rhogvy_pl=vy_pl, rhogvz=vz, rhogvz_pl=vz_pl)
            ica.adjoint_record(dt, nsteps, every, S, F)
            fctx.ica, fctx.F = ica, F
            return S["rhog"], S["rhog_pl"], S["rhogq"], S["rhogq_pl"]

        @staticmethod
        def backward(fctx, g_r, g_rp, g_q, g_qp):
            z = torch.zeros_like
            a = {"rhog": g_r.contiguous().clone(), "rhog_pl": g_rp.contiguous().clone(),
                 "rhogq": g_q.contiguous().clone(), "rhogq_pl": g_qp.contiguous().clone()}
            aw = {k: z(fctx.F[k]) for k in WIND}
            fctx.ica.adjoint_sweep(fctx.F, a, aw)
            return (None, None, None, None, None, a["rhog"], a["rhog_pl"], a["rhogq"], a["rhogq_pl"],
                    aw["rhogvx"], aw["rhogvx_pl"], aw["rhogvy"], aw["rhogvy_pl"], aw["rhogvz"], aw["rhogvz_pl"])

    c = case(5, 0, 24, 3)
    g, f = c["grid"], c["fields"]
    dt = c["dt"]
    dv = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
    S0 = {k: dv(v) for k, v in _noisy(c["state"]).items()}
    F0 = {k: dv(v) for k, v in f.items()}
    ctx = _ctx_dev(g)
    try:
        leaves = {k: v.clone().requires_grad_(True) for k, v in S0.items()}
        wl = {k: F0[k].clone().requires_grad_(True) for k in WIND}
        out = Advect.apply(ctx, dt, 8, 4, {k: F0[k] for k in ("rhogw", "rhogw_pl")}, leaves["rhog"],
                           leaves["rhog_pl"], leaves["rhogq"], leaves["rhogq_pl"], wl["rhogvx"], wl["rhogvx_pl"],
                           wl["rhogvy"], wl["rhogvy_pl"], wl["rhogvz"], wl["rhogvz_pl"])
        r, rp, Q, Qp = out
        _, mask, _ = _objective_seed(g, {"rhog": r.detach(), "rhog_pl": rp.detach(), "rhogq": Q.detach(),
                                         "rhogq_pl": Qp.detach()})
        q = Q / r[None]
        J = (q * q)[:, mask].sum()
        J.backward()
        _, _, _, a, aw = _sweep(ctx, dt, 8, 4, S0, F0)
        for k in STATE:
            _close(leaves[k].grad.cpu().numpy(), a[k].cpu().numpy(), 1e-12, k)
        for k in WIND:
            _close(wl[k].grad.cpu().numpy(), aw[k].cpu().numpy(), 1e-12, k)
    finally:
        ctx.close()
