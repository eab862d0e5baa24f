"""Sub-sampled face fractions of an arbitrary level set (the static CuSolidLevelSet3D::GetFrac)
against the reference's golden fixtures and the FP64 oracle.  The fraction of a cut face is a count
of 128 x 128 sub-face samples; a sample whose interpolated level set lies within rounding of zero
may fall on either side, so two results may differ by a few samples (1/16384 each)."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from test_gpu_parity import N, T

pytestmark = pytest.mark.gpu

SAMPLE = 1.0 / 16384


def _frac(wp, ls, n, h):
    s = wp.mac_shapes3d(*n)
    out = [torch.full(s[k], -1.0, device="cuda") for k in ("xv", "yv", "zv")]
    lso = wp.CuSolidLevelSet3D(n, h)
    lso.GetFrac(*out, ls=T(ls), dim=n, dx=h)
    torch.cuda.synchronize()
    return [N(t) for t in out]


def test_subsampled_fractions_match_reference(wp):
    g = load_golden("frac3d_sub")
    for key in [k for k in g.files if k.startswith("n_")]:
        tag = key[2:]
        n = tuple(int(v) for v in g[key])
        got = _frac(wp, g[f"ls_{tag}"], n, 1.0 / n[0])
        for k, o in zip(("ax", "ay", "az"), got):
            ref = g[f"{k}_{tag}"]
            d = np.abs(o - ref)
            assert d.max() <= 3 * SAMPLE and np.count_nonzero(d) <= max(3, ref.size // 10000), (tag, k, d.max())
            assert np.any((ref > 0) & (ref < 1))


def test_subsampled_fractions_match_oracle_at_64(wp, oracle):
    n = (64, 48, 40)
    h = 1.0 / 64
    rng = np.random.default_rng(3)
    sdf = oracle.sdf_spheres3d(n, h, rng.uniform(0.2, 0.6, (5, 3)), rng.uniform(0.08, 0.2, 5))
    ls = (-sdf).astype(np.float32).astype(np.float64)  # fluid inside the balls
    ref = oracle.fractions3d_subsampled(ls, n, h)
    got = _frac(wp, ls, n, h)
    for r, o in zip(ref, got):
        d = np.abs(o - r)
        assert d.max() <= 3 * SAMPLE and np.count_nonzero(d) <= max(3, r.size // 10000), d.max()
        assert np.all((o >= 0) & (o <= 1))
