"""ica_horizontal_limiter_thuburn_noalloc, the limiter entry point that allocates no
device memory, against ica_horizontal_limiter_thuburn_dev, both called through the
C ABI on device buffers.  Both run the same kernels in the same order, so the test
tolerance is zero: every output equal bit for bit, on two calls in a row.  The file
name sorts last, so in a full run it also runs after every other test of the process."""
import ctypes as C

import numpy as np
import pytest

from cases import case

pytestmark = pytest.mark.gpu
GLEVEL, RLEVEL, KALL = 5, 0, 42


@pytest.fixture(scope="module")
def setup(built, cuda):
    from icoatmosbenchmark_v1_b200 import api
    c = case(GLEVEL, RLEVEL, KALL)
    ctx = api.IcoAdv(GLEVEL, RLEVEL, KALL - 2)
    g = c["geo"]
    ctx.set_geometry(*[g[k] for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                                      "GMTR_a", "GMTR_a_pl")])
    yield c, ctx
    ctx.close()


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _outputs(c):
    import torch
    L, G = c["grid"].lall, c["grid"].gall
    return [_dev(c["qa"]), _dev(c["qa_pl"]), torch.full((2, L, KALL, G), float("nan"), dtype=torch.float64,
                                                         device="cuda"),
            torch.full((2, 2, KALL, 6), float("nan"), dtype=torch.float64, device="cuda")]


def _call(ctx, name, outs, ins, post):
    import torch
    from icoatmosbenchmark_v1_b200 import api
    P = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    qa, qa_pl, qo, qo_pl = outs
    rc = getattr(api.lib(), name)(ctx.h, P(qa), P(qa_pl), *[P(t) for t in ins], P(qo), P(qo_pl),
                                  P(post[0]), P(post[1]))
    torch.cuda.synchronize()
    assert rc == 0, api.lib().ica_last_error().decode()
    return [t.cpu().numpy() for t in outs]


@pytest.mark.parametrize("mode", ["exchange", "snapshot"])
def test_noalloc_limiter_equals_dev_entry_twice(setup, mode):
    import torch
    c, ctx = setup
    ins = [_dev(c[k]) for k in ("q", "q_pl", "d", "d_pl", "ch", "ch_pl", "cm", "cm_pl")]
    post = (None, None)
    if mode == "snapshot":  # Qout after the halo fill, as the extracted kernel reads it
        o = _outputs(c)
        _call(ctx, "ica_horizontal_limiter_thuburn_dev", o, ins, (None, None))
        ctx.COMM_data_transfer(o[2], o[3])
        post = (o[2], o[3])
    ref = _call(ctx, "ica_horizontal_limiter_thuburn_dev", _outputs(c), ins, post)
    first, second = _outputs(c), _outputs(c)  # every device buffer exists before the measured calls
    torch.cuda.synchronize()
    got1 = _call(ctx, "ica_horizontal_limiter_thuburn_noalloc", first, ins, post)
    free1 = torch.cuda.mem_get_info()[0]
    got2 = _call(ctx, "ica_horizontal_limiter_thuburn_noalloc", second, ins, post)
    free2 = torch.cuda.mem_get_info()[0]
    for got in (got1, got2):
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
    assert free2 == free1  # the second call took no device memory


def test_noalloc_rejects_grid_beyond_fixed_scratch(built, cuda):
    from icoatmosbenchmark_v1_b200 import api
    # glevel 6, rlevel 0, kall 52: 66*66 * 52 * 10 = 2,265,120 cells > ICA_NOALLOC_MAX_CELLS
    ctx = api.IcoAdv(6, 0, 50)
    try:
        t = _dev(np.zeros(8))
        p = C.c_void_p(t.data_ptr())
        rc = api.lib().ica_horizontal_limiter_thuburn_noalloc(ctx.h, *([p] * 12), None, None)
        assert rc == -1  # ICA_ERR_ARG
        assert "fixed scratch" in api.lib().ica_last_error().decode()
    finally:
        ctx.close()
