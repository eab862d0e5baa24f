"""Coefficient truncation of a potential (CuWaveletPotentialRecover3D::CutCoefficients) against the
reference's golden fixtures and the FP64 oracle."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from test_gpu_parity import N, T, TOL32

pytestmark = pytest.mark.gpu


def err(ref, got, inp):
    """Deviation relative to the input component: a deep cut leaves little of the potential, and
    the FP32 rounding of the transforms scales with what went in."""
    return float(np.linalg.norm(np.asarray(got, np.float64) - ref) / np.linalg.norm(inp))


def _walls_zero(q):
    qx, qy, qz = (np.array(a) for a in q)
    qx[:, :, [0, -1]] = 0
    qx[[0, -1]] = 0
    qy[:, [0, -1], :] = 0
    qy[[0, -1]] = 0
    qz[:, [0, -1], :] = 0
    qz[:, :, [0, -1]] = 0
    return qx, qy, qz


def test_cut_matches_reference_at_every_level(wp):
    g = load_golden("cut3d")
    for key in [k for k in g.files if k.startswith("n_")]:
        tag = key[2:]
        n = tuple(int(v) for v in g[key])
        rec = wp.CuWaveletPotentialRecover3D(n, 1.0 / n[0])
        q = [T(g[f"{k}_{tag}"]) for k in ("qx", "qy", "qz")]
        for level in range(int(np.log2(min(n))) + 1):
            out = [torch.full_like(t, 5.0) for t in q]
            rec.CutCoefficients(*out, *q, level)
            torch.cuda.synchronize()
            for k, o in zip(("qx", "qy", "qz"), out):
                ref = g[f"{k}_{tag}_cut{level}"]
                e = err(ref, N(o), g[f"{k}_{tag}"])
                assert e < TOL32, (tag, level, k, e)
        rec.close()


@pytest.mark.parametrize("n,level", [((64, 64, 64), 2), ((32, 128, 64), 3), ((64, 32, 16), 4)])
def test_cut_matches_oracle_in_place(wp, oracle, n, level):
    """In place (outputs alias the inputs) at sizes past the fixtures, against the FP64 oracle."""
    s = oracle.mac_shapes3d(*n)
    rng = np.random.default_rng(level)
    q = _walls_zero([rng.standard_normal(s[k]).astype(np.float32).astype(np.float64) for k in ("qx", "qy", "qz")])
    ref = oracle.cut3d(*q, n, level)
    rec = wp.CuWaveletPotentialRecover3D(n, 1.0 / n[0])
    t = [T(a) for a in q]
    rec.CutCoefficients(*t, *t, level)
    torch.cuda.synchronize()
    for r, o, a in zip(ref, t, q):
        assert err(r, N(o), a) < TOL32
    with pytest.raises(wp.WPError):
        rec.CutCoefficients(*t, *t, int(np.log2(min(n))) + 1)
    rec.close()
