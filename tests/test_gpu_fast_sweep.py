"""Eikonal redistancing (CuFastSweeping::Solve / ReinitLevelSet) against the reference's fixed point
and the FP64 oracle's iterates (both run the same deterministic iteration)."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from test_gpu_parity import N, T

pytestmark = pytest.mark.gpu


def test_fast_sweep_matches_reference_fixed_point(wp):
    g = load_golden("fsweep")
    n = tuple(int(v) for v in g["n"])
    for mode, fn in (("reinit", wp.CuFastSweeping.ReinitLevelSet), ("solve", wp.CuFastSweeping.Solve)):
        ls = T(g["ls_" + mode])
        fn(ls, n, float(g["h"]), int(g["iters"]))
        torch.cuda.synchronize()
        ref = g["out_" + mode]
        assert np.abs(N(ls) - ref).max() <= 2e-6 * np.abs(ref).max(), mode


@pytest.mark.parametrize("iters", [1, 3, 40])
def test_fast_sweep_iterates_match_oracle(wp, oracle, iters):
    """Every iterate, not only the fixed point: the GPU runs the oracle's Jacobi iteration."""
    n = (40, 36, 28)
    h = 1.0 / 40
    sdf = oracle.sdf_spheres3d(n, h, [[0.4, 0.5, 0.45], [0.7, 0.3, 0.6]], [0.2, 0.12])
    ls = (0.7 * sdf).astype(np.float32).astype(np.float64)
    ref = oracle.fast_sweep(ls, n, h, iters, True)
    t = T(ls)
    wp.CuFastSweeping.ReinitLevelSet(t, n, h, iters)
    torch.cuda.synchronize()
    # FP32 storage between iterations: at most one rounding per iteration, not amplified (the update
    # is monotone and non-expansive)
    assert np.abs(N(t) - ref).max() <= 1e-5 * np.abs(ref).max()


def test_particles_to_ls_matches_reference_fixed_point(wp):
    g = load_golden("fsweep")
    n = tuple(int(v) for v in g["n"])
    ls = torch.empty((n[2], n[0], n[1]), device="cuda")
    x = T(g["particles"])
    wp.CuFastSweeping.ParticlesToLs(ls, x, n, float(g["h"]), float(g["radius"]), float(g["max_dis"]),
                                    int(g["iters"]))
    torch.cuda.synchronize()
    ref = g["out_particles"]
    assert np.abs(N(ls) - ref).max() <= 1e-5 * np.abs(ref).max()
    assert np.array_equal(N(ls) > 0, ref > 0)
