"""CPU tests of the oracle: pinned against the reference's golden vectors
(communication self-test logs) and checked for the properties the restated
kernels and the composed step must have."""
import json
from pathlib import Path

import numpy as np
import pytest

import comm_tables as T
from cases import case, interior, vertical_inputs

GOLDEN = Path(__file__).parent / "golden" / "comm_gl04rl00_2rank.json"


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


def test_comm_golden_tables_2rank(O):
    """COMM_debugtest of the reference (gl4 rl0 vlayer 20, 2 ranks): initial labels,
    after COMM_data_transfer and after COMM_var, both ranks, bit for bit."""
    fx = json.loads(GOLDEN.read_text())
    t = O.Topo(4, 0, 2)
    assert t.rellist_nmax(1) == 320 and t.rellist_nmax(2) == 320  # "*** rellist_nmax: 320"
    kall, kmin, kmax = 22, 2, 21
    sgp = lambda p, l: O.lib().orc_topo_have_sgp(t.h, p, l)
    var, vpl = T.debugtest_init(2, t.lall, t.gall_1d, kall, kmin, kmax, t.rgnid, sgp)

    def check(phase):
        for r in range(2):
            got = T.tables(var[r], vpl[r], kmin, t.gall_1d, t.lall)
            assert got == fx["ranks"][r][phase], (phase, r)

    check("init")
    t.data_transfer(var, vpl)
    check("comm")
    T.set_pole_halo_labels(var, 2, t.lall, t.gall_1d, kmin, kmax, t.rgnid, t.vert_num())
    t.comm_var(var, vpl)
    check("polefill")


def test_region_topology_matches_log(O):
    """Edge and vertex links printed in msg.pe000000 (lines 73-140) for regions 1-5."""
    t = O.Topo(4, 0, 2)
    et = t.edge_tab()
    assert et[0].tolist() == [[6, 3], [5, 3], [2, 2], [10, 2]]  # (1,SW)->(6,NE) (1,NW)->(5,NE) ...
    assert et[4].tolist() == [[7, 3], [4, 3], [1, 2], [6, 2]]
    vn = t.vert_num()
    assert vn[0].tolist() == [3, 5, 3, 3]
    assert t.rgn4pl(1) == 1 and t.rgn4pl(2) == 6


@pytest.mark.parametrize("glevel,rlevel", [(3, 0), (4, 1), (5, 2)])
def test_comm_single_vs_multi_rank_interior(O, glevel, rlevel):
    """Region halos after the transfer do not depend on the number of ranks (only the
    south-pole ring order does, see test_topology); checked on random data."""
    t1 = O.Topo(glevel, rlevel, 1)
    t2 = O.Topo(glevel, rlevel, 2)
    rng = np.random.default_rng(1)
    v = rng.standard_normal((2, t1.lall, 3, t1.gall))
    vp = rng.standard_normal((2, 2, 3, 6))
    a, ap = v.copy(), vp.copy()
    t1.data_transfer([a], [ap])
    half = t1.lall // 2
    b = [v[:, :half].copy(), v[:, half:].copy()]
    bp = [vp.copy(), vp.copy()]
    t2.data_transfer(b, bp)
    np.testing.assert_array_equal(np.concatenate(b, 1), a)


def test_flux_constant_state_zero_divergence(O):
    """Zero wind gives zero flux and GRD_xc == GRD_xr on every face the flux loops reach."""
    c = case(4, 0, 6)
    g, d = c["grid"], c["dims"]
    z = np.zeros_like(c["fields"]["rhog"])
    zp = np.zeros_like(c["fields"]["rhog_pl"])
    flx, flx_pl, xc, xc_pl = O.horizontal_flux(d, g.have_sgp, c["fields"]["rhog"], c["fields"]["rhog_pl"],
                                               z, zp, z, zp, z, zp, 600.0, c["geo"])
    assert np.all(flx == 0) and np.all(flx_pl == 0)
    m = g.interior_mask()
    for a in range(3):
        for x in range(3):
            got = xc[x, a].transpose(1, 0, 2)[:, m]
            ref = np.broadcast_to(c["geo"]["GRD_xr"][x, a][m], got.shape)
            np.testing.assert_array_equal(got, ref)


def test_flux_antisymmetry(O):
    """flx_h(ij,1)*area(ij) == -flx_h(ip1j,4)*area(ip1j) (one face, two cells) to rounding."""
    c = case(4, 0, 6)
    g, flx = c["grid"], c["flx"]
    area = c["geo"]["GMTR_p"][0]
    G = g.gall_1d
    m = g.interior_mask()
    ij = np.nonzero(m[0])[0]
    ij = ij[(ij % G) < g.gmax - 1]  # ip1j interior too
    a = flx[0][:, :, ij] * area[:, None, ij]
    b = -flx[3][:, :, ij + 1] * area[:, None, ij + 1]
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_limiter_keeps_faces_within_bounds(O):
    """After the Thuburn limiter every face value lies within the min/max of its upwind stencil."""
    c = case(4, 0, 6)
    g, d = c["grid"], c["dims"]
    qa, qa_pl, qo, qo_pl = O.horizontal_limiter(d, g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"],
                                                np.zeros_like(c["q"]), np.zeros_like(c["q_pl"]), c["ch"],
                                                c["ch_pl"], c["cm"], c["cm_pl"], topo=c["topo"])
    q = c["q"]
    qi = interior(qa, g)[..., 1:-1, :]
    assert qi.min() >= q.min() - 1e-12
    assert qi.max() <= q.max() + 1e-12
    assert np.any(qa != c["qa"])  # the limiter did clip something


def test_limiter_snapshot_mode_equals_exchange_mode(O):
    """Feeding Qout_post = COMM(Qout_prev) reproduces the original NICAM (exchange) mode."""
    c = case(4, 0, 6)
    g, d = c["grid"], c["dims"]
    args = (d, g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], c["d"], c["d_pl"], c["ch"], c["ch_pl"],
            c["cm"], c["cm_pl"])
    a1, ap1, qo, qop = O.horizontal_limiter(*args, topo=c["topo"])
    post, postp = qo.copy(), qop.copy()
    c["topo"].data_transfer([post], [postp])
    a2, ap2, qo2, qop2 = O.horizontal_limiter(*args, Qout_post=post, Qout_post_pl=postp)
    np.testing.assert_array_equal(a1, a2)
    np.testing.assert_array_equal(ap1, ap2)
    np.testing.assert_array_equal(qo, qo2)


def test_vertical_limiter_monotone(O):
    c = case(4, 0, 10)
    d = c["dims"]
    qh, qh_pl, ck, ck_pl = vertical_inputs(c)
    out, out_pl = O.vertical_limiter(d, qh, qh_pl, c["q"], c["q_pl"], np.zeros_like(c["q"]),
                                     np.zeros_like(c["q_pl"]), ck, ck_pl)
    lo = np.minimum(c["q"][:, :-1], c["q"][:, 1:])
    hi = np.maximum(c["q"][:, :-1], c["q"][:, 1:])
    inner = out[:, 2:-1]
    assert np.all(inner >= lo[:, 1:-1] - 1e-12) and np.all(inner <= hi[:, 1:-1] + 1e-12)


def test_composed_step_properties(O):
    """Mass conservation, monotonicity and constancy of the composed step (unpinned rows)."""
    c = case(4, 0, 8, ntr=2)
    g, d = c["grid"], c["dims"]
    S = {k: v.copy() for k, v in c["state"].items()}
    S["rhogq"] = np.concatenate([S["rhogq"], 0.7 * S["rhog"][None]], 0).copy()
    S["rhogq_pl"] = np.concatenate([S["rhogq_pl"], 0.7 * S["rhog_pl"][None]], 0).copy()
    m = g.interior_mask()
    kk = slice(g.kmin - 1, g.kmax)
    area, dz = g.arrays["GMTR_p"][0], g.arrays["dz"]

    def mass(S):
        a = (S["rhogq"][:, :, kk] * area[None, :, None] * dz[None, None, kk, None] * m[None, :, None]).sum((1, 2, 3))
        return a + (S["rhogq_pl"][:, :, kk, 0] * g.arrays["GMTR_p_pl"][0][None, :, 0, None]
                    * dz[None, None, kk]).sum((1, 2))

    m0 = mass(S)
    qmin, qmax = (S["rhogq"] / S["rhog"]).min(), (S["rhogq"] / S["rhog"]).max()
    for _ in range(3):
        O.step(d, g.have_sgp, c["topo"], c["dt"], S, c["fields"], g.arrays, nthreads=4)
    assert np.all(np.abs(mass(S) - m0) <= 1e-13 * np.abs(m0))
    q = S["rhogq"] / S["rhog"]
    assert q[:2].min() >= qmin - 1e-12 and q[:2].max() <= qmax + 1e-12
    assert np.abs(interior(q[2], g)[kk] - 0.7).max() < 1e-13
