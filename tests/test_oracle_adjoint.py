"""The oracle's adjoint of the composed step (oracle/oracle_adjoint.c, the FP64 reference
gradient) against central finite differences of the oracle's forward step.

J = sum of seeded random weights times the state after n steps.  Components are drawn
from rhogq, rhog and the three wind components (regions and pole centres); a component
whose one-sided differences disagree is at a limiter kink and is skipped.  The tracer
fields get seeded noise of 1e-3 relative: the slotted cylinder's flat regions are exact
ties of every min/max/clamp (value = bound = 0), where the forward's branch is a
subgradient that coordinate differences cannot see."""
import numpy as np
import pytest

from cases import case

WIND = ("rhogvx", "rhogvx_pl", "rhogvy", "rhogvy_pl", "rhogvz", "rhogvz_pl")


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


@pytest.mark.parametrize("glevel,rlevel,kall,ntr,nsteps", [(3, 0, 6, 2, 2), (3, 1, 8, 1, 1)])
def test_oracle_adjoint_against_finite_differences(O, glevel, rlevel, kall, ntr, nsteps):
    c = case(glevel, rlevel, kall, ntr)
    g, f, d, topo, geo = c["grid"], c["fields"], c["dims"], c["topo"], c["grid"].arrays
    rng = np.random.default_rng(11)
    S0 = {k: v.copy() for k, v in c["state"].items()}
    S0["rhogq"] = S0["rhogq"] + 1e-3 * S0["rhog"][None] * rng.random(S0["rhogq"].shape)
    S0["rhogq_pl"] = S0["rhogq_pl"] + 1e-3 * S0["rhog_pl"][None] * rng.random(S0["rhogq_pl"].shape)
    w = {k: rng.standard_normal(v.shape) for k, v in S0.items()}

    def J(S, F):
        S = {k: v.copy() for k, v in S.items()}
        for _ in range(nsteps):
            O.step(d, g.have_sgp, topo, c["dt"], S, F, geo, nthreads=4)
        return sum(float((w[k] * S[k]).sum()) for k in S)

    states = [S0]
    for _ in range(nsteps):
        S = {k: v.copy() for k, v in states[-1].items()}
        O.step(d, g.have_sgp, topo, c["dt"], S, f, geo, nthreads=4)
        states.append(S)
    adj = {k: w[k].copy() for k in S0}
    aw = {k: np.zeros_like(f[k]) for k in WIND}
    for s in range(nsteps - 1, -1, -1):
        O.step_adjoint(d, g.have_sgp, topo, c["dt"], states[s], f, geo, adj, aw)
    J0 = J(S0, f)
    checked = 0
    for n in range(36):
        which = ["rhogq", "rhog", "rhogvx", "rhogvy", "rhogvz", "rhogq_pl"][n % 6]
        arr = S0[which] if which in S0 else f[which]
        while True:
            idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
            if which.endswith("_pl"):
                idx = idx[:-1] + (0,)
                ok = True
            else:
                p, G = idx[-1], g.gall_1d
                i, j = p % G + 1, p // G + 1
                ok = g.gmin <= i <= g.gmax and g.gmin <= j <= g.gmax
            if ok and 1 <= idx[-2] <= kall - 2:
                break
        grad = adj[which][idx] if which in adj else aw[which][idx]
        h = 1e-6 * max(1.0, abs(arr[idx]))
        vals = []
        for sgn in (1, -1):
            if which in S0:
                S = {k: v.copy() for k, v in S0.items()}
                S[which][idx] += sgn * h
                vals.append(J(S, f))
            else:
                F = dict(f)
                F[which] = f[which].copy()
                F[which][idx] += sgn * h
                vals.append(J(S0, F))
        right, left = (vals[0] - J0) / h, (J0 - vals[1]) / h
        if abs(right - left) > 1e-4 * max(abs(right), abs(left), 1e-6):
            continue  # limiter kink within the step
        fd = (vals[0] - vals[1]) / (2 * h)
        tol = max(1e-5 * abs(fd), 1e-6 * max(abs(fd), 1.0) + 2e-9 * abs(J0) / h)
        assert abs(grad - fd) <= tol, (which, idx, grad, fd)
        checked += 1
    assert checked >= 25
