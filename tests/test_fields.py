"""The synthetic tracer fields of the uneven-batch configuration: half of the tracers are
seeded random fields of real spherical harmonics of degree <= 16, clipped to [0, 1]."""
import numpy as np
import torch


def _basis(lmax, th, ph):
    import scipy.special as sp
    cols = []
    for l in range(lmax + 1):
        for m in range(l + 1):
            Y = sp.sph_harm_y(l, m, th, ph)
            cols.append(Y.real)
            if m > 0:
                cols.append(Y.imag)
    return np.stack(cols, 1)


def test_smooth_tracer_is_spherical_harmonic_degree_16():
    """Before clipping, the field is exactly a combination of degree <= 16 harmonics (a least-squares
    fit with that basis leaves FP64 rounding) and needs degree 16 (the degree <= 15 fit does not)."""
    from icoatmosbenchmark_v1_b200.fields import spherical_harmonic_field
    rng = np.random.default_rng(7)
    v = rng.standard_normal((3, 1500))
    v /= np.linalg.norm(v, axis=0)
    f = spherical_harmonic_field(torch.as_tensor(v), seed=20261204).numpy()
    th, ph = np.arccos(v[2]), np.arctan2(v[1], v[0])
    res = {}
    for lmax in (15, 16):
        B = _basis(lmax, th, ph)
        c = np.linalg.lstsq(B, f, rcond=None)[0]
        res[lmax] = np.abs(B @ c - f).max() / np.abs(f).max()
    assert res[16] < 1e-12
    assert res[15] > 1e-3


def test_mixed_tracers_in_unit_interval_and_seeded():
    from icoatmosbenchmark_v1_b200 import fields as F
    from icoatmosbenchmark_v1_b200.grid import Grid
    g = Grid(3, 0, 6)
    q, qp = F.tracer_mixing_ratio(g, 4, "mixed")
    q2, _ = F.tracer_mixing_ratio(g, 4, "mixed")
    assert torch.equal(q, q2)
    assert float(q.min()) >= 0.0 and float(q.max()) <= 1.0
    assert float(qp.min()) >= 0.0 and float(qp.max()) <= 1.0
    assert float(q[0].std()) > 0.05  # the smooth tracer varies
