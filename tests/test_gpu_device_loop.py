"""The device-side cycle loop of the mixed-precision tolerance solve (a CUDA graph with a while-node)
against the host-driven loop, and the per-row uniform-fraction fast path of the column kernels
against the oracle."""
import numpy as np
import pytest
import torch

from test_gpu_parity import N, T, _sphere_problem

pytestmark = pytest.mark.gpu


def _solve(wp, mg, f, host_loop, **kw):
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, f, precision=wp.PREC_MIXED, raise_on_fail=False, host_loop=host_loop, **kw)
    torch.cuda.synchronize()
    return rep, N(dst), mg.Iterate64()


def _same(a, b):
    """Same status and cycle count; residual history, FP32 result and FP64 iterate equal up to the
    order of the atomic FP64 sums (the active mean and the defect norms), which differs between any
    two solves, host loop or not."""
    ra, da, pa = a
    rb, db, pb = b
    assert ra["status"] == rb["status"] and ra["cycles"] == rb["cycles"], (ra, rb)
    np.testing.assert_allclose(ra["rel_residual"], rb["rel_residual"], rtol=1e-9)
    np.testing.assert_allclose(ra["history"], rb["history"], rtol=1e-9)
    scale = np.abs(pb).max()
    assert np.abs(pa - pb).max() <= 1e-12 * scale and np.abs(da - db).max() <= 1e-6 * scale


@pytest.mark.parametrize("start", [0, 1])
@pytest.mark.parametrize("tol,cap", [(1e-10, 60), (1e-13, 3), (0.0, 4), (1e-10, 1)])
def test_device_loop_matches_host_loop(wp, oracle, start, tol, cap):
    """The device loop stops where the host loop stops: the converged case, the cycle cap reached
    first, a fixed cycle count and a single cycle."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 64, seed=21, spheres=([[0.3, 0.4, 0.5], [0.7, 0.6, 0.5]], [0.15, 0.1]))
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    tf = T(f)
    kw = dict(rel_tol=tol, max_cycles=cap, start=start)
    dev = _solve(wp, mg, tf, False, **kw)
    host = _solve(wp, mg, tf, True, **kw)
    _same(dev, host)
    # the cached graph replays for a second solve on the same right-hand side
    _same(_solve(wp, mg, tf, False, **kw), host)
    if tol == 1e-13:
        assert dev[0]["status"] == "WP_ERR_NOT_CONVERGED" and dev[0]["cycles"] == cap


def test_device_loop_follows_new_inputs_and_tiles(wp, oracle):
    """The captured graph is rebuilt for a new right-hand-side buffer, a new cycle shape and a new
    tile choice; an in-place change of the same buffer is read by the replay."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32, seed=4)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    f1 = T(f)
    f2 = T(f[::-1].copy())
    kw = dict(rel_tol=1e-10, max_cycles=60)
    for fx in (f1, f2, f1):
        _same(_solve(wp, mg, fx, False, **kw), _solve(wp, mg, fx, True, **kw))
    f1.mul_(-0.5)
    _same(_solve(wp, mg, f1, False, **kw), _solve(wp, mg, f1, True, **kw))
    kw2 = dict(rel_tol=1e-10, max_cycles=60, nu1=1, nu2=3, start=1)
    _same(_solve(wp, mg, f1, False, **kw2), _solve(wp, mg, f1, True, **kw2))
    mg.SetTile(0, 0, 3, 2)
    _same(_solve(wp, mg, f1, False, **kw), _solve(wp, mg, f1, True, **kw))


@pytest.mark.parametrize("case", ["fluid", "box", "spheres"])
def test_uniform_rows_match_oracle_per_cycle(wp, oracle, case):
    """Rows whose faces are all open skip the fraction loads: FP64 cycles still follow the oracle
    when every row is uniform, next to a box whose faces cut cells part-way, and around spheres."""
    n = 32
    nn = (n, n, n)
    h = 1.0 / n
    if case == "spheres":
        nn, h, a, _, f = _sphere_problem(wp, oracle, n, seed=6, spheres=([[0.5, 0.5, 0.5], [0.2, 0.8, 0.3]], [0.2, 0.1]))
    else:
        from waveletpotentials_b200 import fields
        sdf = np.full((n, n, n), 1.0)
        if case == "box":
            sdf = oracle.sdf_boxes3d(sdf, nn, h, [[0.3 + 0.5 * h, 0.25, 0.4]], [[0.6 + 0.5 * h, 0.55 + 0.5 * h, 0.7]])
        r32 = lambda x: x.astype(np.float32).astype(np.float64)
        a = tuple(r32(x) for x in oracle.fractions3d(sdf, nn, h))
        u = tuple(r32(x) for x in fields.velocity3d(nn, 8))
        f = r32(oracle.divergence3d(*u, *a, nn, (h,) * 3))
    if case == "box":
        assert all(np.any((x > 0.0) & (x < 1.0)) and np.any(x == 0.0) for x in a)
    _, ohist = oracle.mgfrac3d_solve(f, *a, nn, (h,) * 3, 6, 2, 2, 2 / 3, prolong=oracle.PROLONG_TRILINEAR)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    uni, rows = mg.UniformRows(0)
    assert rows == n * n and (uni == rows if case == "fluid" else 0 < uni < rows)
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, T(f), rel_tol=0.0, max_cycles=6, precision=wp.PREC_FP64)
    np.testing.assert_allclose(rep["history"], ohist, rtol=1e-6)
    # the FP32 path (quad sweeps, restriction and the shared-memory coarse cycle) follows as well
    dst32 = torch.zeros(f.shape, device="cuda")
    rep32 = mg.SolveTol(dst32, None, T(f), rel_tol=0.0, max_cycles=6, precision=wp.PREC_FP32)
    np.testing.assert_allclose(rep32["history"][:4], ohist[:4], rtol=1e-3)


@pytest.mark.parametrize("start", [0, 1])
def test_inner_cycles_reach_tolerance_on_both_loops(wp, oracle, start):
    """Two FP32 V-cycles per refinement step: the oracle's FP64 residual meets the tolerance, the
    cycle count is even and within two of the one-cycle schedule's, the history has one entry per
    step, and the device and host loops agree."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 64, seed=23)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    tf = T(f)
    one = _solve(wp, mg, tf, False, rel_tol=1e-10, max_cycles=60, start=start)
    dev = _solve(wp, mg, tf, False, rel_tol=1e-10, max_cycles=60, start=start, inner_cycles=2)
    host = _solve(wp, mg, tf, True, rel_tol=1e-10, max_cycles=60, start=start, inner_cycles=2)
    _same(dev, host)
    rep = dev[0]
    assert rep["status"] == "WP_OK" and rep["cycles"] % 2 == 0 and len(rep["history"]) == rep["cycles"] // 2
    assert one[0]["cycles"] <= rep["cycles"] <= one[0]["cycles"] + 2
    from test_gpu_parity import active_cells
    act = active_cells(*a)
    fc = f.copy()
    fc[act] -= f[act].mean()
    _, r = oracle.frac_residual3d(dev[2], fc, *a, nn, (h,) * 3)
    assert np.linalg.norm(r) / np.linalg.norm(f) <= 1.5e-10


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_persistent_coarse_levels_match_launch_by_launch(wp, oracle, precision):
    """The levels below the finest run as one cooperative launch (phases with grid barriers) or
    launch by launch: the same cycles (FP32 contraction order aside), the same tolerance reached,
    on the device loop and on the host loop."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 128, seed=31, spheres=([[0.4, 0.5, 0.45], [0.7, 0.3, 0.6]], [0.18, 0.1]))
    prec = wp.PREC_FP32 if precision == "fp32" else wp.PREC_MIXED
    tf = T(f)
    outs = []
    for on, host_loop in ((0, False), (1, False), (1, True)):
        mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
        mg.SetTile(0, 3, 0, on)
        dst = torch.zeros(f.shape, device="cuda")
        kw = dict(rel_tol=0.0, max_cycles=5) if precision == "fp32" else dict(rel_tol=1e-10, max_cycles=60)
        rep = mg.SolveTol(dst, None, tf, precision=prec, raise_on_fail=False, host_loop=host_loop, **kw)
        torch.cuda.synchronize()
        outs.append((rep, N(dst)))
    for rep, d in outs[1:]:
        assert rep["status"] == outs[0][0]["status"] and rep["cycles"] == outs[0][0]["cycles"]
        np.testing.assert_allclose(rep["history"], outs[0][0]["history"], rtol=1e-4 if precision == "fp32" else 1e-6)
        scale = np.abs(outs[0][1]).max()
        assert np.abs(d - outs[0][1]).max() <= 1e-4 * scale
