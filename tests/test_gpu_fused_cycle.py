"""The fused finest-level V(2,2) cycle (pre-smoothing + residual restriction in one pass,
prolongation + post-smoothing in another, wp_mg_fused.cuh) against the same cycle run one kernel per
sweep and transfer, and its tolerance solves checked in FP64 by the oracle."""
import numpy as np
import pytest
import torch

from test_gpu_parity import N, T, _sphere_problem

pytestmark = pytest.mark.gpu


def _problem(wp, oracle, nn, seed, spheres, d=None):
    from waveletpotentials_b200 import fields
    h = 1.0 / max(nn)
    d = d or (h, h, h)
    sdf = oracle.sdf_spheres3d(nn, h, *spheres)
    r32 = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
    a = [r32(x) for x in oracle.fractions3d(sdf, nn, h)]
    u = [r32(x) for x in fields.velocity3d(nn, seed)]
    f = r32(oracle.divergence3d(*u, *a, nn, d))
    return a, f, d


def _no_mean(d, ref):
    """d without its mean over the active cells (the Neumann problem's null space: rounding moves
    the constant component of the iterate freely; fully solid cells stay 0)."""
    act = ref != 0
    out = d.copy()
    out[act] -= d[act].mean()
    return out


def _solve(wp, mg, f, fused, precision, zc=0, **kw):
    mg.SetTile(0, 4, zc, 1 if fused else 0)
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, f, precision=precision, raise_on_fail=False, **kw)
    torch.cuda.synchronize()
    p64 = mg.Iterate64() if precision != wp.PREC_FP32 else None
    return rep, N(dst), p64


CASES = {
    "cube64": ((64, 64, 64), 3, ([[0.5, 0.5, 0.5], [0.2, 0.75, 0.3]], [0.2, 0.1])),
    # spheres cut by the walls and tiles of every kind; extents of unequal tile counts per axis
    "box96x64x48": ((96, 64, 48), 5, ([[0.05, 0.5, 0.3], [0.7, 0.02, 0.45], [0.5, 0.5, 0.0]], [0.12, 0.1, 0.15])),
    "fluid32": ((32, 32, 32), 7, ([[5.0, 5.0, 5.0]], [0.1])),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_fused_cycle_matches_unfused(wp, oracle, case, precision):
    """Same cycle counts and residual histories and the same iterate to FP32 rounding (the fused
    kernels multiply by a precomputed w / diagonal on uniform planes where the one-sweep kernels
    divide)."""
    nn, seed, sph = CASES[case]
    a, f, d = _problem(wp, oracle, nn, seed, sph)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, d)
    tf = T(f)
    prec = wp.PREC_MIXED if precision == "mixed" else wp.PREC_FP32
    kw = dict(rel_tol=1e-10 if precision == "mixed" else 1e-5, max_cycles=60, inner_cycles=2)
    ra, da, pa = _solve(wp, mg, tf, True, prec, **kw)
    rb, db, pb = _solve(wp, mg, tf, False, prec, **kw)
    assert ra["status"] == rb["status"] == "WP_OK", (ra, rb)
    assert ra["cycles"] == rb["cycles"]
    # FP32 iterates: the histories part at FP32 rounding (1e-8 of ||f||) as they near its floor
    np.testing.assert_allclose(ra["history"], rb["history"], rtol=1e-4, atol=0 if pa is not None else 2e-8)
    scale = np.abs(db).max()
    assert np.abs(_no_mean(da - db, db)).max() <= 1e-5 * scale
    if pa is not None:
        assert np.abs(_no_mean(pa - pb, pb)).max() <= 1e-8 * np.abs(pb).max()
        rel, _ = oracle.frac_residual3d(pa, f, *a, nn, d)
        assert rel <= 1e-10 * 1.5


@pytest.mark.parametrize("zc", [2, 6, 16, 0])
def test_fused_cycle_chunking_is_exact(wp, oracle, zc):
    """The z-chunk of a CTA changes where the pipelines start, never a value: bitwise the same
    iterate for every chunk."""
    nn, seed, sph = CASES["box96x64x48"]
    a, f, d = _problem(wp, oracle, nn, seed, sph)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, d)
    tf = T(f)
    kw = dict(rel_tol=0.0, max_cycles=4, inner_cycles=1)
    ref = _solve(wp, mg, tf, True, wp.PREC_FP32, zc=48, **kw)[1]
    got = _solve(wp, mg, tf, True, wp.PREC_FP32, zc=zc, **kw)[1]
    assert np.array_equal(ref, got)


def test_fused_cycle_anisotropic_spacing(wp, oracle):
    """Unequal spacings per axis: the restriction weights and stencil factors of every axis."""
    nn = (64, 32, 32)
    a, f, d = _problem(wp, oracle, nn, 11, ([[0.4, 0.5, 0.6]], [0.18]), d=(1 / 64, 1.3 / 32, 0.8 / 32))
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, d)
    tf = T(f)
    kw = dict(rel_tol=1e-10, max_cycles=80, inner_cycles=2)
    ra, _, pa = _solve(wp, mg, tf, True, wp.PREC_MIXED, **kw)
    rb, _, pb = _solve(wp, mg, tf, False, wp.PREC_MIXED, **kw)
    assert ra["status"] == "WP_OK" and ra["cycles"] == rb["cycles"]
    assert np.abs(_no_mean(pa - pb, pb)).max() <= 1e-8 * np.abs(pb).max()
    rel, _ = oracle.frac_residual3d(pa, f, *a, nn, d)
    assert rel <= 1.5e-10
