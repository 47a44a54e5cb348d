"""Kernel snapshots in the reference drivers' binary format (dumpio.c): the reader and writer
on CPU, and, on the GPU, the library run on snapshots whose expected outputs the oracle
wrote.  The snapshots are synthetic: region 0 of a glevel-4 grid (gall_1d 18) with the poles,
the form of the drivers' one-region-per-process snapshots at a small size."""
import numpy as np
import pytest

from cases import case
from icoatmosbenchmark_v1_b200 import snapshot as S

DIMS = S.SnapshotDims(gall_1d=18, kall=8)


def _one_region(a):
    """Region 0 of a [..., L, K, G] array."""
    return np.ascontiguousarray(np.asarray(a)[..., :1, :, :])


def _geo_one_region(a, pole):
    """A library geometry array ([..., L, G] or pole [..., LP, P]) in the driver's form with
    the K0 axis: [..., L, 1, G]."""
    a = np.asarray(a)
    if not pole:
        a = a[..., :1, :]
    return np.ascontiguousarray(a[..., None, :])


def synthetic_snapshots(tmp_path, O, zero_d=False):
    """Writes the three drivers' snapshots from oracle outputs; returns {kernel: path}.
    zero_d: the limiters' d = 0, as the composed step passes it."""
    c = dict(case(4, 0, 8, 1))
    if zero_d:
        c["d"], c["d_pl"] = np.zeros_like(c["d"]), np.zeros_like(c["d_pl"])
    g, d, f = c["grid"], c["dims"], c["fields"]
    paths = {}

    arr = dict(flx_h=_one_region(c["flx"]), flx_h_pl=c["flx_pl"], GRD_xc=_one_region(c["xc"]), GRD_xc_pl=c["xc_pl"],
               rho=_one_region(f["rhog"]), rho_pl=f["rhog_pl"])
    for v in ("x", "y", "z"):
        arr[f"rhov{v}"] = _one_region(f[f"rhogv{v}"])
        arr[f"rhov{v}_pl"] = f[f"rhogv{v}_pl"]
    for k, v in c["geo"].items():
        arr[k] = _geo_one_region(v, k.endswith("_pl"))
    paths["dyn_horiz_adv_flux"] = tmp_path / S.file_name("dyn_horiz_adv_flux")
    S.write_snapshot("dyn_horiz_adv_flux", paths["dyn_horiz_adv_flux"], arr, DIMS)

    args = (d, g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], c["d"], c["d_pl"], c["ch"], c["ch_pl"],
            c["cm"], c["cm_pl"])
    qa, qa_pl, qo, qo_pl = O.horizontal_limiter(*args, topo=c["topo"])
    post, post_pl = qo.copy(), qo_pl.copy()
    c["topo"].data_transfer([post], [post_pl])
    arr = dict(q_a_prev=_one_region(c["qa"]), q_a_prev_pl=c["qa_pl"], q_a=_one_region(qa), q_a_pl=qa_pl,
               q=_one_region(c["q"]), q_pl=c["q_pl"], d=_one_region(c["d"]), d_pl=c["d_pl"],
               ch=_one_region(c["ch"]), ch_pl=c["ch_pl"], cmask=_one_region(c["cm"]), cmask_pl=c["cm_pl"],
               Qout_prev=_one_region(qo), Qout_prev_pl=qo_pl, Qout_post=_one_region(post), Qout_post_pl=post_pl)
    paths["dyn_horiz_adv_limiter"] = tmp_path / S.file_name("dyn_horiz_adv_limiter")
    S.write_snapshot("dyn_horiz_adv_limiter", paths["dyn_horiz_adv_limiter"], arr, DIMS)

    from cases import vertical_inputs
    qh, qh_pl, ck, ck_pl = vertical_inputs(c)
    rqh, rqh_pl = O.vertical_limiter(d, qh, qh_pl, c["q"], c["q_pl"], c["d"], c["d_pl"], ck, ck_pl)
    arr = dict(q_h_prev=_one_region(qh), q_h_prev_pl=qh_pl, q_h=_one_region(rqh), q_h_pl=rqh_pl,
               q=_one_region(c["q"]), q_pl=c["q_pl"], d=_one_region(c["d"]), d_pl=c["d_pl"],
               ck=_one_region(ck), ck_pl=ck_pl)
    paths["dyn_vert_adv_limiter"] = tmp_path / S.file_name("dyn_vert_adv_limiter")
    S.write_snapshot("dyn_vert_adv_limiter", paths["dyn_vert_adv_limiter"], arr, DIMS)
    return paths, c["dt"]


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


def test_reference_snapshot_sizes():
    """The reference's snapshots (gall_1d 130, kall 42, one region and the poles) hold these
    many 8-byte reals: the sums of the drivers' array extents."""
    def nbytes(kernel):
        return 8 * sum(int(np.prod(e)) for _, e, _ in S.layout(kernel))
    G, K, P = 130 * 130, 42, 6
    assert nbytes("dyn_vert_adv_limiter") == 8 * (G * K * (4 + 2) + P * K * 2 * (4 + 2))
    assert nbytes("dyn_horiz_adv_limiter") == 8 * (G * K * (6 * 4 + 1 + 1 + 2 * 2)
                                                   + P * K * 2 * (4 + 1 + 1 + 2 * 2))
    assert nbytes("dyn_horiz_adv_flux") == 8 * (G * K * (6 + 9 + 4) + P * K * 2 * (1 + 3 + 4)
                                                + G * (9 + 8 + 10 + 36) + P * 2 * (3 + 8 + 5 + 18))
    assert S.file_name("dyn_horiz_adv_flux", 3) == "snapshot.dyn_horiz_adv_flux.pe000003"


def test_snapshot_round_trip_big_endian(tmp_path):
    """Arrays come back as written; the file is big-endian float64 in Fortran (column-major)
    order, one array after the other with no record markers."""
    rng = np.random.default_rng(3)
    lay = S.layout("dyn_vert_adv_limiter", DIMS)
    arr = {n: rng.standard_normal(e[::-1]) for n, e, _ in lay}
    p = tmp_path / "snap"
    S.write_snapshot("dyn_vert_adv_limiter", p, arr, DIMS)
    raw = p.read_bytes()
    assert len(raw) == 8 * sum(a.size for a in arr.values())
    # first array, Fortran order: q_h_prev(ij, k, l) with ij fastest
    first = arr["q_h_prev"]
    assert np.frombuffer(raw[:8], ">f8")[0] == first[0, 0, 0]
    assert np.frombuffer(raw[8:16], ">f8")[0] == first[0, 0, 1]
    assert np.frombuffer(raw[8 * DIMS.gall:8 * DIMS.gall + 8], ">f8")[0] == first[0, 1, 0]
    back = S.read_snapshot("dyn_vert_adv_limiter", p, DIMS)
    assert list(back) == [n for n, _, _ in lay]
    for n in arr:
        np.testing.assert_array_equal(back[n], arr[n])
    with pytest.raises(ValueError):
        S.read_snapshot("dyn_horiz_adv_limiter", p, DIMS)
    with pytest.raises(ValueError):
        S.write_snapshot("dyn_vert_adv_limiter", p, {**arr, "ck": arr["ck"][:1]}, DIMS)


def test_value_check_format():
    """The driver's (1x,A,A16,3(A,ES24.16)) line: 16-character name, each value right-justified
    in 24 characters with 16 digits after the point and a two-digit exponent (three, without
    the E, past 99)."""
    line = S.value_check("check_q_h", np.array([1.0, -2.0, 0.5]))
    assert line == (" +check[check_q_h       ] max=  1.0000000000000000E+00,min= -2.0000000000000000E+00,"
                    "sum= -5.0000000000000000E-01")
    assert S.value_check("d", np.array([-0.0])).split("] ", 1)[1] == \
        "max= -0.0000000000000000E+00,min= -0.0000000000000000E+00,"\
        "sum=  0.0000000000000000E+00"  # a sum starts from +0, as the Fortran SUM does
    assert S._es(3.3842023700197510e-02) == "  3.3842023700197510E-02"
    big = S._es(-2.0 ** -400)  # -3.87e-121: three exponent digits, no E
    assert len(big) == 24 and "E" not in big and big.endswith("-121") and big.startswith(" -3.8725919148493")
    assert len(S.value_check("a_name_longer_than_16", np.ones(2))) == len(S.value_check("x", np.ones(2)))


def test_synthetic_snapshots_read_back(tmp_path, O):
    paths, _ = synthetic_snapshots(tmp_path, O)
    for kernel, p in paths.items():
        s = S.read_snapshot(kernel, p, DIMS)
        assert all(np.isfinite(v).all() for v in s.values())


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", S.KERNELS)
def test_run_snapshot_matches_expected(tmp_path, O, cuda, kernel):
    """The library on a snapshot reproduces the snapshot's expected outputs: bit-exact for the
    flux and the two limiters (FP64 kernels built without contraction)."""
    paths, dt = synthetic_snapshots(tmp_path, O)
    got, diffs = S.run_snapshot(kernel, paths[kernel], DIMS, dt=dt)
    assert list(diffs) == [n for n, _, out in S.layout(kernel, DIMS) if out]
    for name, dv in diffs.items():
        assert np.isfinite(got[name]).all()
        assert np.abs(dv).max() == 0.0, (name, np.abs(dv).max())


class _OracleCtx:
    """Stands in for api.IcoAdv on CPU (same constructor for a driver's arrays, the same
    methods, in-place outputs), computing with the oracle on the driver's one region, so
    that the snapshot plumbing (the driver's sizes, geometry without the K0 axis, the
    driver's initial output values) is checked without a GPU."""

    @classmethod
    def regions(cls, gall_1d, kall, kmin, kmax, lall, have_pl, have_sgp, device=0):
        from oracle import oracle
        self = cls.__new__(cls)
        glevel = int(round(np.log2(gall_1d - 2)))
        self.O = oracle
        self.d = oracle.make_dims(glevel, 0, kall, kmin, kmax, lall=lall, have_pl=int(have_pl))
        self.have_sgp = np.asarray(have_sgp, np.int32)
        self.gall, self.lall = gall_1d * gall_1d, lall
        self.sizes = type("Sizes", (), {"lall": lall})()
        return self

    def set_geometry(self, *geo):
        names = ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl", "GMTR_a", "GMTR_a_pl")
        for n, a in zip(names, geo):  # the library's layout: [..., lall, gall] and [..., 2, 6]
            assert a.shape[-2:] == ((2, 6) if n.endswith("_pl") else (self.lall, self.gall)), (n, a.shape)
        self.geo = dict(zip(names, geo))

    def horizontal_flux(self, flx, flx_pl, xc, xc_pl, rho, rho_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl, dt):
        a, ap, x, xp = self.O.horizontal_flux(self.d, self.have_sgp, rho, rho_pl, vx, vx_pl, vy, vy_pl, vz, vz_pl,
                                              dt, self.geo)
        flx[...], xc[...] = a, x
        flx_pl[:, :, 1:], xc_pl[..., 1:] = ap[:, :, 1:], xp[..., 1:]  # pole centre not written

    def horizontal_limiter_thuburn(self, qa, qa_pl, q, q_pl, d, d_pl, ch, ch_pl, cm, cm_pl, qo, qo_pl, post, post_pl):
        a, ap, o, op = self.O.horizontal_limiter(self.d, self.have_sgp, qa, qa_pl, q, q_pl, d, d_pl, ch, ch_pl, cm,
                                                 cm_pl, Qout_post=post, Qout_post_pl=post_pl)
        qa[...], qa_pl[...], qo[...], qo_pl[...] = a, ap, o, op

    def vertical_limiter_thuburn(self, qh, qh_pl, q, q_pl, d, d_pl, ck, ck_pl):
        a, ap = self.O.vertical_limiter(self.d, qh, qh_pl, q, q_pl, d, d_pl, ck, ck_pl)
        qh[...], qh_pl[...] = a, ap

    def close(self):
        pass


@pytest.mark.parametrize("kernel", S.KERNELS)
def test_run_snapshot_plumbing_with_oracle(tmp_path, O, monkeypatch, kernel):
    """run_snapshot on the driver's one-region arrays, with the oracle in place of the CUDA
    library (the oracle restates the kernels for any ADM_lall): the region's outputs come back
    equal to the expected ones, which the oracle computed on the whole grid."""
    from icoatmosbenchmark_v1_b200 import api
    monkeypatch.setattr(api, "IcoAdv", _OracleCtx)
    paths, dt = synthetic_snapshots(tmp_path, O)
    got, diffs = S.run_snapshot(kernel, paths[kernel], DIMS, dt=dt)
    for name, dv in diffs.items():
        assert got[name].shape == S.read_snapshot(kernel, paths[kernel], DIMS)[name].shape
        assert np.abs(dv).max() == 0.0, (name, np.abs(dv).max())


def test_cli_check_prints_driver_summaries(tmp_path, O, capsys):
    paths, _ = synthetic_snapshots(tmp_path, O)
    S.main(["check", "dyn_vert_adv_limiter", str(paths["dyn_vert_adv_limiter"]), "--gall-1d", "18", "--kall", "8"])
    out = capsys.readouterr().out.splitlines()
    assert out[0].strip() == "### Input ###"
    assert [ln.split("]")[0].split("[")[1].strip() for ln in out[1:]] == \
        [n for n, _, _ in S.layout("dyn_vert_adv_limiter", DIMS)]


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", S.KERNELS)
def test_run_snapshot_single_precision(tmp_path, O, cuda, kernel):
    """The FP32 entry points on the same FP64 snapshots, as the drivers' RP = SP build reads and
    converts them (d = 0): the flux and the limited values within FP32 rounding of the FP64
    expected ones (normwise, the tolerances of the FP32 kernel tests).  Qout is left out: the
    FP32 and FP64 zero-outflow switches differ on ill-conditioned cells."""
    paths, dt = synthetic_snapshots(tmp_path, O, zero_d=True)
    got, diffs = S.run_snapshot(kernel, paths[kernel], DIMS, dt=dt, precision="f32")
    s = S.read_snapshot(kernel, paths[kernel], DIMS)
    tol = 2e-5 if kernel == "dyn_horiz_adv_limiter" else 1e-5
    for name, dv in diffs.items():
        if name.startswith("Qout"):
            continue
        e = np.abs(dv).max() / max(np.abs(s[name]).max(), 1e-30)
        assert e <= tol, (name, e)


def test_cli_run_prints_zero_diffs_with_oracle(tmp_path, O, monkeypatch, capsys):
    """`run`: the input summaries, the outputs and the driver's point-by-point diff lines, here
    with the oracle in the library's place (all diffs zero)."""
    from icoatmosbenchmark_v1_b200 import api
    monkeypatch.setattr(api, "IcoAdv", _OracleCtx)
    paths, dt = synthetic_snapshots(tmp_path, O)
    S.main(["run", "dyn_horiz_adv_flux", str(paths["dyn_horiz_adv_flux"]), "--gall-1d", "18", "--kall", "8",
            "--dt", repr(dt)])
    out = capsys.readouterr().out.splitlines()
    i = out.index(" ### Validation : point-by-point diff ###")
    diff = out[i + 1:]
    assert [ln.split("[")[1].split("]")[0].strip() for ln in diff] == \
        ["check_flx_h", "check_flx_h_pl", "check_GRD_xc", "check_GRD_xc_pl"]
    zero = S._es(0.0)
    for ln in diff:
        assert ln.endswith(f"max={zero},min={zero},sum={zero}"), ln  # x - x is +0
