"""The C ABI as a reference driver uses it: tests/c_driver/ica_driver.c, a plain-C program built
with gcc against libicoadv.so, holds one region of a glevel-7 grid with both poles (the drivers'
130 x 130 x 42 x 1 arrays, ADM_lall = 1) and calls ica_init_regions, ica_set_geometry and the
three kernel entry points on host arrays.  On the GPU its outputs equal the oracle's bit for
bit; the oracle runs on the same one-region arrays (its kernels take any ADM_lall), and on that
region they equal its whole-grid run."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "icoatmosbenchmark_v1_b200"
GL, KALL = 7, 42  # gall_1d 130


def _compile(built, out):
    gcc = shutil.which("gcc") or "gcc"
    cmd = [gcc, "-O2", "-Wall", "-Werror", "-std=c11", f"-I{ROOT / 'include'}", str(ROOT / "tests/c_driver/ica_driver.c"),
           f"-L{PKG}", "-licoadv", f"-Wl,-rpath,{PKG}", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_driver_builds_and_links(built, tmp_path):
    """The plain-C driver compiles against include/icoadv.h and links to the library (no GPU)."""
    exe = _compile(built, tmp_path / "ica_driver")
    assert exe.exists()


def _region0(a):
    return np.ascontiguousarray(np.asarray(a)[..., :1, :, :])


def _geo0(a, pole):
    a = np.asarray(a)
    return np.ascontiguousarray(a if pole else a[..., :1, :])


@pytest.mark.gpu
def test_driver_one_region_gl7_k42_bit_exact(built, cuda, tmp_path):
    from cases import case, vertical_inputs
    from oracle import oracle as O
    exe = _compile(built, tmp_path / "ica_driver")
    c = case(GL, 0, KALL, 1)
    g, f, dt = c["grid"], c["fields"], c["dt"]
    d1 = O.make_dims(GL, 0, KALL, lall=1, have_pl=1)
    sgp1 = np.ones(1, np.int32)
    geo1 = {k: _geo0(v, k.endswith("_pl")) for k, v in c["geo"].items()}
    A = dict(geo1)
    # flux: the output arrays start from arbitrary values (the drivers start from their snapshot's)
    rng = np.random.default_rng(3)
    A.update(rho=_region0(f["rhog"]), rho_pl=f["rhog_pl"])
    for v in "xyz":
        A[f"rhov{v}"] = _region0(f[f"rhogv{v}"])
        A[f"rhov{v}_pl"] = f[f"rhogv{v}_pl"]
    A.update(flx_h=rng.random(_region0(c["flx"]).shape), flx_h_pl=rng.random(c["flx_pl"].shape),
             GRD_xc=rng.random(_region0(c["xc"]).shape), GRD_xc_pl=rng.random(c["xc_pl"].shape))
    # limiter: Qout after the whole grid's halo fill, as the driver's snapshot holds it
    _, _, qo, qo_pl = O.horizontal_limiter(c["dims"], g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], c["d"],
                                           c["d_pl"], c["ch"], c["ch_pl"], c["cm"], c["cm_pl"], topo=c["topo"])
    post, post_pl = qo.copy(), qo_pl.copy()
    c["topo"].data_transfer([post], [post_pl])
    A.update(q_a=_region0(c["qa"]), q_a_pl=c["qa_pl"], q=_region0(c["q"]), q_pl=c["q_pl"], d=_region0(c["d"]),
             d_pl=c["d_pl"], ch=_region0(c["ch"]), ch_pl=c["ch_pl"], cmask=_region0(c["cm"]), cmask_pl=c["cm_pl"],
             Qout_post=_region0(post), Qout_post_pl=post_pl)
    qh, qh_pl, ck, ck_pl = vertical_inputs(c)
    A.update(q_h=_region0(qh), q_h_pl=qh_pl, vq=_region0(c["q"]), vq_pl=c["q_pl"], vd=_region0(c["d"]),
             vd_pl=c["d_pl"], ck=_region0(ck), ck_pl=ck_pl)
    for k, v in A.items():
        np.ascontiguousarray(v, np.float64).tofile(tmp_path / f"{k}.f64")
    env = dict(os.environ)
    r = subprocess.run([str(exe), str(tmp_path), str(g.gall_1d), str(KALL), repr(float(dt))], capture_output=True,
                       text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = lambda n, like: np.fromfile(tmp_path / f"out_{n}.f64").reshape(np.shape(like))  # noqa: E731

    # the oracle on the driver's one region
    flx, flx_pl, xc, xc_pl = O.horizontal_flux(d1, sgp1, A["rho"], A["rho_pl"], A["rhovx"], A["rhovx_pl"],
                                               A["rhovy"], A["rhovy_pl"], A["rhovz"], A["rhovz_pl"], dt, geo1)
    qa1, qa1_pl, qo1, qo1_pl = O.horizontal_limiter(d1, sgp1, A["q_a"], A["q_a_pl"], A["q"], A["q_pl"], A["d"],
                                                    A["d_pl"], A["ch"], A["ch_pl"], A["cmask"], A["cmask_pl"],
                                                    Qout_post=A["Qout_post"], Qout_post_pl=A["Qout_post_pl"])
    qh1, qh1_pl = O.vertical_limiter(d1, A["q_h"], A["q_h_pl"], A["vq"], A["vq_pl"], A["vd"], A["vd_pl"], A["ck"],
                                     A["ck_pl"])
    # ... which on that region is its whole-grid run
    np.testing.assert_array_equal(flx, _region0(c["flx"]))
    np.testing.assert_array_equal(xc, _region0(c["xc"]))
    qaw, _, _, _ = O.horizontal_limiter(c["dims"], g.have_sgp, c["qa"], c["qa_pl"], c["q"], c["q_pl"], c["d"],
                                        c["d_pl"], c["ch"], c["ch_pl"], c["cm"], c["cm_pl"], Qout_post=post,
                                        Qout_post_pl=post_pl)
    np.testing.assert_array_equal(qa1, _region0(qaw))
    # the driver's outputs, bit for bit (the pole centres of flx_h_pl / GRD_xc_pl are not written
    # by the kernel and keep the driver's values)
    np.testing.assert_array_equal(got("flx_h", flx), flx)
    np.testing.assert_array_equal(got("GRD_xc", xc), xc)
    fp = got("flx_h_pl", flx_pl)
    np.testing.assert_array_equal(fp[..., 1:], flx_pl[..., 1:])
    np.testing.assert_array_equal(fp[..., 0], A["flx_h_pl"][..., 0])
    xp = got("GRD_xc_pl", xc_pl)
    np.testing.assert_array_equal(xp[..., 1:], xc_pl[..., 1:])
    for n, ref in (("q_a", qa1), ("q_a_pl", qa1_pl), ("Qout_prev", qo1), ("Qout_prev_pl", qo1_pl), ("q_h", qh1),
                   ("q_h_pl", qh1_pl)):
        np.testing.assert_array_equal(got(n, ref), ref, err_msg=n)
    assert "ica_driver ok" in r.stdout
