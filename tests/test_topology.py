"""CPU tests of the product's host side: the composed single-GPU halo/pole plan
against the oracle and the reference's golden tables, and the C ABI library
(loads, exports every declared symbol, rejects bad arguments without a GPU)."""
import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import comm_tables as T

GOLDEN = Path(__file__).parent / "golden" / "comm_gl04rl00_2rank.json"


@pytest.fixture(scope="module")
def api(built):
    from icoatmosbenchmark_v1_b200 import api
    return api


@pytest.fixture(scope="module")
def O(built):
    from oracle import oracle
    return oracle


@pytest.mark.parametrize("glevel,rlevel", [(2, 0), (4, 0), (5, 0), (3, 1), (4, 1), (5, 2), (6, 2)])
@pytest.mark.parametrize("pole_fill", [False, True])
def test_plan_equals_sequential_transfer(api, O, glevel, rlevel, pole_fill):
    """The composed gather reproduces COMM_data_transfer / COMM_var of one process bit for bit."""
    t = O.Topo(glevel, rlevel, 1)
    rng = np.random.default_rng(glevel * 10 + rlevel)
    v = rng.standard_normal((3, t.lall, 4, t.gall))
    vp = rng.standard_normal((3, 2, 4, 6))
    a, ap = v.copy(), vp.copy()
    (t.comm_var if pole_fill else t.data_transfer)([a], [ap])
    api.apply_plan_numpy(api.comm_plan(glevel, rlevel, pole_fill), v, vp)
    np.testing.assert_array_equal(v, a)
    np.testing.assert_array_equal(vp, ap)


@pytest.mark.parametrize("glevel,rlevel", [(4, 0), (5, 1), (6, 2)])
def test_plan_is_race_free_and_in_bounds(api, glevel, rlevel):
    dst, src = api.comm_plan(glevel, rlevel, True)
    npt = 10 * 4 ** rlevel * (2 ** (glevel - rlevel) + 2) ** 2 + 12
    assert dst.min() >= 0 and dst.max() < npt and src.min() >= 0 and src.max() < npt
    assert len(np.unique(dst)) == len(dst)
    assert not np.intersect1d(dst, src).size


def test_plan_vs_golden_2rank_tables(api, O):
    """The reference's 2-rank self-test, redone with the single-process plan, gives the same
    tables except the south-pole ring: there the reference's r2p message is packed in region
    order and unpacked in ring order, so the 2-rank run permutes the ring (rank 1 log, slots 2-6
    = regions 9,8,7,6,10); one process (and the GPU) puts region r at its ring slot (10,9,8,7,6)."""
    fx = json.loads(GOLDEN.read_text())
    t = O.Topo(4, 0, 2)
    kall, kmin, kmax = 22, 2, 21
    sgp = lambda p, l: O.lib().orc_topo_have_sgp(t.h, p, l)
    var, vpl = T.debugtest_init(2, t.lall, t.gall_1d, kall, kmin, kmax, t.rgnid, sgp)
    v = np.concatenate(var, 1)
    vp = vpl[0].copy()
    api.apply_plan_numpy(api.comm_plan(4, 0, False), v, vp)
    for r in range(2):
        got = T.tables(v[:, 5 * r:5 * r + 5], vp if r == 0 else vpl[1], kmin, t.gall_1d, 5)
        exp = fx["ranks"][r]["comm"]
        assert got["prc_rgn"] == exp["prc_rgn"] and got["ij"] == exp["ij"]
        if r == 0:
            assert got["pole_prc_rgn"][0] == exp["pole_prc_rgn"][0]  # north ring: identical
            assert [p[1] for p in got["pole_prc_rgn"][1][1:]] == [10, 9, 8, 7, 6]
            assert [p[1] for p in exp["pole_prc_rgn"][1][1:]] == [9, 8, 7, 6, 10]


def test_topology_info(api, O):
    for gl, rl in [(4, 0), (5, 1), (5, 2)]:
        sgp, r4, ring = api.topology_info(gl, rl)
        t = O.Topo(gl, rl, 1)
        np.testing.assert_array_equal(sgp, t.have_sgp())
        assert list(r4) == [t.rgn4pl(1), t.rgn4pl(2)]


def test_library_exports_every_declared_symbol(api):
    names = api.exported_symbols()
    assert len(names) >= 24
    out = subprocess.run(["nm", "-D", "--defined-only", str(api.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = api.lib()
    for n in names:
        assert hasattr(lib, n)


def test_host_entry_points_reject_bad_arguments(api):
    lib = api.lib()
    assert lib.ica_comm_plan(0, 0, 0, C.byref(C.c_int()), None, None) == -1
    assert lib.ica_comm_plan(4, 5, 0, C.byref(C.c_int()), None, None) == -1
    assert lib.ica_init(None, None) == -1
    d = api.Dims(4, 0, 0, 0)  # vlayer 0
    h = C.c_void_p()
    assert lib.ica_init(C.byref(d), C.byref(h)) == -1
    assert lib.ica_finalize(None) == -1
    # NULL context on every kernel entry point
    assert lib.ica_horizontal_flux(None, *([None] * 12), C.c_double(1.0)) == -1
    assert lib.ica_comm_data_transfer(None, None, None, 1, 1) == -1


def test_init_without_gpu_reports_error(api):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = api.Dims(4, 0, 20, 0)
    h = C.c_void_p()
    rc = api.lib().ica_init(C.byref(d), C.byref(h))
    assert rc == -3 and not h.value  # ICA_ERR_CUDA, no context
    assert api.lib().ica_last_error()


@pytest.mark.parametrize("gl,rl", [(3, 0), (4, 1)])
def test_grid_from_oracle_tables_equals_grid_from_library(built, gl, rl):
    """The synthetic grid built with the oracle's topology and halo plan (the reference arm's
    grid) is the grid the library's host tables give, array for array."""
    from icoatmosbenchmark_v1_b200.grid import Grid
    from oracle import oracle as O
    a = Grid(gl, rl, 6)
    b = Grid(gl, rl, 6, tables=O.GridTables())
    assert np.array_equal(a.have_sgp, b.have_sgp)
    assert set(a.arrays) == set(b.arrays)
    for k in a.arrays:
        assert np.array_equal(a.arrays[k], b.arrays[k]), k
