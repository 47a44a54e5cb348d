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


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from cases import case
from icoatmosbenchmark_v1_b200 import api
c = case(5, 0, 42)
ctx = api.IcoAdv(5, 0, 40)
g = c["geo"]
ctx.set_geometry(*[g[k] for k in ("GRD_xr", "GRD_xr_pl", "GMTR_p", "GMTR_p_pl", "GMTR_t", "GMTR_t_pl",
                                  "GMTR_a", "GMTR_a_pl")])
D = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
ins = [D(c[k]) for k in ("q", "q_pl", "d", "d_pl", "ch", "ch_pl", "cm", "cm_pl")]
outs = [[D(c["qa"]), D(c["qa_pl"]), D(np.zeros((2,) + c["q"].shape)), D(np.zeros((2, 2, 42, 6)))] for _ in range(2)]
P = lambda t: C.c_void_p(t.data_ptr())
L = api.lib()
# the same kernels through the allocating entry point first: their code is loaded and
# that entry point's own scratch allocated before the measurement
assert L.ica_horizontal_limiter_thuburn_dev(ctx.h, P(outs[0][0]), P(outs[0][1]), *map(P, ins), P(outs[0][2]),
                                            P(outs[0][3]), None, None) == 0
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
assert L.ica_horizontal_limiter_thuburn_noalloc(ctx.h, P(outs[1][0]), P(outs[1][1]), *map(P, ins), P(outs[1][2]),
                                                P(outs[1][3]), None, None) == 0, L.ica_last_error()
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
for a, b in zip(outs[0], outs[1]):
    assert torch.equal(a, b)
print("FREE", free0, free1)
ctx.close()
"""


def test_noalloc_first_call_in_fresh_process_takes_no_memory(built):
    """The first noalloc call of a process: its fixed array was loaded by ica_init, so the
    GPU's free memory is the same before and after that call."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, ICOADV_NO_BUILD="1")
    r = subprocess.run([sys.executable, "-c", _FRESH, str(root)], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("FREE")][-1].split()
    assert int(line[1]) == int(line[2]), line
