"""GPU parity of the reference-interface kernels against the oracle, through
the C ABI (host-pointer entry points, which copy in, launch and copy out).

FP64: the kernels are built without FMA contraction and keep the reference's
operation order, so they must equal the oracle bit for bit (the test also
states the 1e-12 relative bound the path is specified to).  FP32 (RP = SP):
within 1e-5 normwise relative error of the FP64 oracle (the limiters with d = 0,
the value the composed step passes).  Halo/pole fills: bit-exact."""
import numpy as np
import pytest

from cases import case, qout_mask, rel_err, vertical_inputs

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-12
FP32_TOL = 1e-5
# The FP32 limiter divides by the outflow Courant sum; fed FP32-rounded inputs (6e-8) its output
# is conditioned a few times worse than the other kernels, so it gets 2e-5.
FP32_LIMITER_TOL = 2e-5
CONFIGS = [(5, 0, 42), (4, 1, 10), (3, 0, 5)]


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


@pytest.fixture(scope="module")
def ctxs(built, cuda):
    from icoatmosbenchmark_v1_b200 import api
    out = {}
    yield out
    for c in out.values():
        c.close()


def ctx_for(ctxs, glevel, rlevel, kall, geo):
    from icoatmosbenchmark_v1_b200 import api
    key = (glevel, rlevel, kall)
    if key not in ctxs:
        c = api.IcoAdv(glevel, rlevel, kall - 2)
        c.set_geometry(*[geo[k] for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                                          "GMTR_a", "GMTR_a_pl")])
        ctxs[key] = c
    return ctxs[key]


def assert_fp64_parity(got, ref):
    assert rel_err(got, ref) <= FP64_TOL
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("glevel,rlevel,kall", CONFIGS)
def test_horizontal_flux_fp64(O, ctxs, glevel, rlevel, kall):
    c = case(glevel, rlevel, kall)
    f = c["fields"]
    ctx = ctx_for(ctxs, glevel, rlevel, kall, c["geo"])
    G, L, K = c["grid"].gall, c["grid"].lall, kall
    flx = np.full((6, L, K, G), np.nan)
    flx_pl = np.zeros((2, K, 6))
    xc = np.full((3, 3, L, K, G), np.nan)
    xc_pl = np.zeros((3, 2, K, 6))
    ctx.horizontal_flux(flx, flx_pl, xc, xc_pl, f["rhog"], f["rhog_pl"], f["rhogvx"], f["rhogvx_pl"],
                        f["rhogvy"], f["rhogvy_pl"], f["rhogvz"], f["rhogvz_pl"], c["dt"])
    assert_fp64_parity(flx, c["flx"])
    assert_fp64_parity(xc, c["xc"])
    assert_fp64_parity(flx_pl[:, :, 1:], c["flx_pl"][:, :, 1:])
    assert_fp64_parity(xc_pl[..., 1:], c["xc_pl"][..., 1:])


def test_horizontal_flux_fp32(O, ctxs):
    c = case(5, 0, 42)
    f = c["fields"]
    ctx = ctx_for(ctxs, 5, 0, 42, c["geo"])
    G, L, K = c["grid"].gall, c["grid"].lall, 42
    s = lambda a: np.ascontiguousarray(a, np.float32)
    flx = np.zeros((6, L, K, G), np.float32)
    flx_pl = np.zeros((2, K, 6), np.float32)
    xc = np.zeros((3, 3, L, K, G), np.float32)
    xc_pl = np.zeros((3, 2, K, 6), np.float32)
    ctx.horizontal_flux(flx, flx_pl, xc, xc_pl, s(f["rhog"]), s(f["rhog_pl"]), s(f["rhogvx"]), s(f["rhogvx_pl"]),
                        s(f["rhogvy"]), s(f["rhogvy_pl"]), s(f["rhogvz"]), s(f["rhogvz_pl"]), c["dt"])
    assert rel_err(flx, c["flx"]) <= FP32_TOL
    assert rel_err(xc, c["xc"]) <= FP32_TOL
    assert rel_err(flx_pl[:, :, 1:], c["flx_pl"][:, :, 1:]) <= FP32_TOL


@pytest.mark.parametrize("glevel,rlevel,kall", CONFIGS)
@pytest.mark.parametrize("mode", ["snapshot", "exchange"])
def test_horizontal_limiter_fp64(O, ctxs, glevel, rlevel, kall, mode):
    c = case(glevel, rlevel, kall)
    g, d = c["grid"], c["dims"]
    ctx = ctx_for(ctxs, glevel, rlevel, kall, c["geo"])
    args = (d, g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], c["d"], c["d_pl"], c["ch"], c["ch_pl"],
            c["cm"], c["cm_pl"])
    ra, rap, rqo, rqop = O.horizontal_limiter(*args, topo=c["topo"])
    post = postp = None
    if mode == "snapshot":  # the extracted kernel's input Qout_post = COMM(Qout_prev)
        post, postp = rqo.copy(), rqop.copy()
        c["topo"].data_transfer([post], [postp])
    qa, qa_pl = c["qa"].copy(), c["qa_pl"].copy()
    qo = np.full_like(rqo, np.nan)
    qop = np.full_like(rqop, np.nan)
    ctx.horizontal_limiter_thuburn(qa, qa_pl, c["q"], c["q_pl"], c["d"], c["d_pl"], c["ch"], c["ch_pl"], c["cm"],
                                   c["cm_pl"], qo, qop, post, postp)
    assert_fp64_parity(qa, ra)
    assert_fp64_parity(qa_pl, rap)
    assert_fp64_parity(qo, rqo)
    assert_fp64_parity(qop, rqop)


def test_horizontal_limiter_fp32(O, ctxs):
    """d = 0, as the composed step passes it.  q_a everywhere; Qout on the cells whose
    outflow bounds are well conditioned (cases.qout_mask)."""
    c = case(5, 0, 42)
    g, d = c["grid"], c["dims"]
    ctx = ctx_for(ctxs, 5, 0, 42, c["geo"])
    z, z_pl = np.zeros_like(c["d"]), np.zeros_like(c["d_pl"])
    ra, rap, rqo, rqop = O.horizontal_limiter(d, g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], z, z_pl,
                                              c["ch"], c["ch_pl"], c["cm"], c["cm_pl"], topo=c["topo"])
    s = lambda a: np.ascontiguousarray(a, np.float32)
    qa, qa_pl = s(c["qa"]), s(c["qa_pl"])
    qo, qop = np.zeros(rqo.shape, np.float32), np.zeros(rqop.shape, np.float32)
    ctx.horizontal_limiter_thuburn(qa, qa_pl, s(c["q"]), s(c["q_pl"]), s(z), s(z_pl), s(c["ch"]), s(c["ch_pl"]),
                                   s(c["cm"]), s(c["cm_pl"]), qo, qop)
    assert rel_err(qa, ra) <= FP32_LIMITER_TOL and rel_err(qa_pl, rap) <= FP32_LIMITER_TOL
    m, m_pl = qout_mask(c["ch"], c["ch_pl"])
    assert m.mean() > 0.95
    assert rel_err(qo[:, m], rqo[:, m]) <= FP32_LIMITER_TOL
    assert rel_err(qop[:, m_pl, 0], rqop[:, m_pl, 0]) <= FP32_LIMITER_TOL


@pytest.mark.parametrize("glevel,rlevel,kall", CONFIGS)
def test_vertical_limiter_fp64(O, ctxs, glevel, rlevel, kall):
    c = case(glevel, rlevel, kall)
    d = c["dims"]
    ctx = ctx_for(ctxs, glevel, rlevel, kall, c["geo"])
    qh, qh_pl, ck, ck_pl = vertical_inputs(c)
    ref, ref_pl = O.vertical_limiter(d, qh, qh_pl, c["q"], c["q_pl"], c["d"], c["d_pl"], ck, ck_pl)
    a, ap = qh.copy(), qh_pl.copy()
    ctx.vertical_limiter_thuburn(a, ap, c["q"], c["q_pl"], c["d"], c["d_pl"], ck, ck_pl)
    assert_fp64_parity(a, ref)
    assert_fp64_parity(ap, ref_pl)


def test_vertical_limiter_fp32(O, ctxs):
    c = case(5, 0, 42)
    ctx = ctx_for(ctxs, 5, 0, 42, c["geo"])
    qh, qh_pl, ck, ck_pl = vertical_inputs(c)
    z, z_pl = np.zeros_like(c["d"]), np.zeros_like(c["d_pl"])  # d = 0, as the composed step passes it
    ref, ref_pl = O.vertical_limiter(c["dims"], qh, qh_pl, c["q"], c["q_pl"], z, z_pl, ck, ck_pl)
    s = lambda a: np.ascontiguousarray(a, np.float32)
    a, ap = s(qh), s(qh_pl)
    ctx.vertical_limiter_thuburn(a, ap, s(c["q"]), s(c["q_pl"]), s(z), s(z_pl), s(ck), s(ck_pl))
    assert rel_err(a, ref) <= FP32_TOL and rel_err(ap, ref_pl) <= FP32_TOL


@pytest.mark.parametrize("glevel,rlevel,kall", CONFIGS)
@pytest.mark.parametrize("vmax", [1, 4])
def test_comm_data_transfer_and_var_bit_exact(O, ctxs, glevel, rlevel, kall, vmax):
    c = case(glevel, rlevel, kall)
    ctx = ctx_for(ctxs, glevel, rlevel, kall, c["geo"])
    rng = np.random.default_rng(vmax)
    L, G = c["grid"].lall, c["grid"].gall
    v = rng.standard_normal((vmax, L, kall, G))
    vp = rng.standard_normal((vmax, 2, kall, 6))
    for fn, ofn in ((ctx.COMM_data_transfer, c["topo"].data_transfer), (ctx.COMM_var, c["topo"].comm_var)):
        a, ap = v.copy(), vp.copy()
        ofn([a], [ap])
        b, bp = v.copy(), vp.copy()
        fn(b, bp)
        np.testing.assert_array_equal(b, a)
        np.testing.assert_array_equal(bp, ap)


def test_comm_golden_tables_on_gpu(O, ctxs):
    """COMM_debugtest of the reference, gl4 rl0, one process on the GPU: region tables of both
    logs bit for bit; the pole rings in single-process order (see test_topology)."""
    import json
    from pathlib import Path

    import comm_tables as T
    from icoatmosbenchmark_v1_b200 import api
    fx = json.loads((Path(__file__).parent / "golden" / "comm_gl04rl00_2rank.json").read_text())
    t = O.Topo(4, 0, 2)
    sgp = lambda p, l: O.lib().orc_topo_have_sgp(t.h, p, l)
    var, vpl = T.debugtest_init(2, t.lall, t.gall_1d, 22, 2, 21, t.rgnid, sgp)
    v = np.ascontiguousarray(np.concatenate(var, 1))
    vp = vpl[0].copy()
    ctx = api.IcoAdv(4, 0, 20)
    try:
        ctx.COMM_data_transfer(v, vp)
        for r in range(2):
            got = T.tables(v[:, 5 * r:5 * r + 5], vp, 2, t.gall_1d, 5)
            exp = fx["ranks"][r]["comm"]
            assert got["prc_rgn"] == exp["prc_rgn"] and got["ij"] == exp["ij"]
        assert T.tables(v[:, :5], vp, 2, t.gall_1d, 5)["pole_ij"][0] == fx["ranks"][0]["comm"]["pole_ij"][0]
    finally:
        ctx.close()


def test_launch_count_and_errors(ctxs):
    from icoatmosbenchmark_v1_b200 import api
    ctx = api.IcoAdv(3, 0, 3)
    try:
        n0 = ctx.launch_count
        v = np.zeros((1, 10, 5, 100))
        vp = np.zeros((1, 2, 5, 6))
        ctx.COMM_data_transfer(v, vp)
        assert ctx.launch_count == n0 + 1
        with pytest.raises(api.IcoAdvError):  # geometry not registered
            z = np.zeros((10, 5, 100))
            zp = np.zeros((2, 5, 6))
            ctx.horizontal_flux(np.zeros((6, 10, 5, 100)), zp.copy(), np.zeros((3, 3, 10, 5, 100)),
                                np.zeros((3, 2, 5, 6)), z, zp, z, zp, z, zp, z, zp, 1.0)
    finally:
        ctx.close()
