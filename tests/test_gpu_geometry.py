"""The grid and its metrics built on the device (ica_grid_build_dev: GMTR_p/t/a_setup and
OPRT_gradient_setup of dyn_metrics, with COMM's halo fills) against the host build of the same
grid (grid.Grid, numpy).  Both round every sum and product the same way; atan2, sin and cos
differ between the CUDA and host math libraries by an ulp, so the bound is 1e-12 of each
array's largest magnitude, not bit equality.  Positions are bisections of unit vectors with
no library math function and come out bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("glevel,rlevel", [(5, 0), (4, 1), (3, 2)])
def test_device_grid_equals_host_grid(built, cuda, glevel, rlevel):
    from icoatmosbenchmark_v1_b200 import api
    from icoatmosbenchmark_v1_b200.grid import Grid
    g = Grid(glevel, rlevel, 6)
    ctx = api.IcoAdv(glevel, rlevel, 4)
    try:
        got = ctx.build_grid(g.R)
        import torch
        torch.cuda.synchronize()
        for k, v in got.items():
            ref = g.arrays[k]
            a = v.cpu().numpy()
            assert a.shape == ref.shape, (k, a.shape, ref.shape)
            scale = max(float(np.abs(ref).max()), 1e-300)
            err = float(np.abs(a - ref).max())
            assert err <= 1e-12 * scale, (k, err, scale)
        np.testing.assert_array_equal(got["GRD_x"].cpu().numpy(), g.arrays["GRD_x"])
        np.testing.assert_array_equal(got["GRD_x_pl"].cpu().numpy(), g.arrays["GRD_x_pl"])
    finally:
        ctx.close()
