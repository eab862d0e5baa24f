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


def test_particles_to_ls_near_walls_matches_oracle(wp, oracle):
    """Particles within half a cell of every wall and in the corners: the rough-distance cells
    that would lie outside the grid are skipped (the reference indexes past the grid there), and
    the GPU agrees with the oracle's FP64 restatement everywhere, with no write outside the grid
    (the guard cells around the level set keep their sentinel)."""
    n = (24, 20, 16)
    h = 1.0 / 24
    ext = np.array([n[0] * h, n[1] * h, n[2] * h])
    e = 0.3 * h
    pts = [[e, 0.5 * ext[1], 0.5 * ext[2]], [ext[0] - e, 0.4 * ext[1], 0.6 * ext[2]],
           [0.5 * ext[0], e, 0.3 * ext[2]], [0.3 * ext[0], ext[1] - e, 0.5 * ext[2]],
           [0.6 * ext[0], 0.5 * ext[1], e], [0.4 * ext[0], 0.6 * ext[1], ext[2] - e],
           [e, e, e], [ext[0] - e, ext[1] - e, ext[2] - e], [e, ext[1] - e, e], [ext[0] - e, e, ext[2] - e],
           [0.5 * ext[0], 0.5 * ext[1], 0.5 * ext[2]]]
    xyz = np.asarray(pts, np.float32).astype(np.float64)
    radius, max_dis, iters = 1.5 * h, 1.0, 60
    ref = oracle.particles_to_ls(xyz, n, h, radius, max_dis, iters)
    cells = n[0] * n[1] * n[2]
    buf = torch.full((cells + 2 * 4096,), 12345.0, device="cuda")
    ls = buf[4096:4096 + cells].view(n[2], n[0], n[1])
    wp.CuFastSweeping.ParticlesToLs(ls, T(xyz), n, h, radius, max_dis, iters)
    torch.cuda.synchronize()
    got = N(ls)
    assert np.all(N(buf[:4096]) == 12345.0) and np.all(N(buf[4096 + cells:]) == 12345.0)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    sure = np.abs(ref) > 1e-6 * np.abs(ref).max()
    assert np.array_equal((got > 0)[sure], (ref > 0)[sure])


@pytest.mark.parametrize("start", ["band", "wavy"])
def test_particles_to_ls_narrow_matches_reference_and_oracle(wp, oracle, start):
    """ParticlesToLsNarrow from the caller's level set: the reference's fixed point (FP32) and, with
    particles also within half a cell of the walls, the oracle (no write outside the grid)."""
    g = load_golden("p2ls_narrow")
    n = tuple(int(v) for v in g["n"])
    h, radius, iters = float(g["h"]), float(g["radius"]), int(g["iters"])
    ls = T(g[start + "_ls"]).contiguous()
    wp.CuFastSweeping.ParticlesToLsNarrow(ls, T(g[start + "_particles"]), n, h, radius, 1.0, iters)
    torch.cuda.synchronize()
    ref = g[start + "_out"]
    assert np.abs(N(ls) - ref).max() <= 1e-5 * np.abs(ref).max()
    assert np.array_equal(N(ls) > 0, ref > 0)
    e = 0.3 * h
    ext = np.array([n[0] * h, n[1] * h, n[2] * h])
    pts = np.concatenate([g[start + "_particles"], [[e, e, e], [ext[0] - e, 0.5 * ext[1], ext[2] - e]]])
    xyz = np.asarray(pts, np.float32).astype(np.float64)
    ref = oracle.particles_to_ls_narrow(g[start + "_ls"], xyz, n, h, radius, iters)
    cells = n[0] * n[1] * n[2]
    buf = torch.full((cells + 2 * 4096,), 12345.0, device="cuda")
    ls = buf[4096:4096 + cells].view(n[2], n[0], n[1])
    ls.copy_(T(g[start + "_ls"]))
    wp.CuFastSweeping.ParticlesToLsNarrow(ls, T(xyz), n, h, radius, 1.0, iters)
    torch.cuda.synchronize()
    assert np.abs(N(ls) - ref).max() <= 1e-5 * np.abs(ref).max()
    assert float(buf[:4096].min()) == 12345.0 and float(buf[4096 + cells:].min()) == 12345.0
