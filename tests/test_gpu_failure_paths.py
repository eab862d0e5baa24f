"""Failure paths reached without a GPU fault: a bounded device wait that runs out (one arrival
withheld by the test-only wp_debug_withhold_wait, so the wait is on a flag that nothing sets), a
non-finite input, and a batch replay whose planned step counts no longer meet the tolerance.  Each
checks the status the call returns and that the next ordinary call on the same handle succeeds with
the result it gave before."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _sphere_case(wp, n, seed=3):
    """Face fractions of one sphere and the divergence of a seeded velocity field on an n^3 grid."""
    from waveletpotentials_b200 import fields
    d = (n, n, n)
    h = 1.0 / n
    s = wp.mac_shapes3d(*d)
    sls = wp.CuSolidLevelSet3D(d, h)
    sls.InitLsSpheres(np.array([[0.5, 0.45, 0.55]]), np.array([0.22]))
    a = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
    sls.GetFrac(*a)
    u = [torch.as_tensor(x, dtype=torch.float32, device="cuda") for x in fields.velocity3d(d, seed=seed)]
    b = torch.empty(s["p"], device="cuda")
    wp.CuConvergence.GetB_3d_frac_vel(b, *u, *a, d, h)
    torch.cuda.synchronize()
    return d, h, a, u, b


def _kernel_names(fn):
    """Kernel classes launched by fn() (the library's own launch accounting)."""
    L = __import__("waveletpotentials_b200._lib", fromlist=["lib"]).lib()
    L.wp_profile_reset()
    L.wp_profile_enable(1)
    try:
        fn()
        torch.cuda.synchronize()
    finally:
        L.wp_profile_enable(0)
    names = []
    for i in range(L.wp_profile_collect()):
        name = ctypes.create_string_buffer(64)
        lc, t, by = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
        L.wp_profile_entry(i, name, 64, ctypes.byref(lc), ctypes.byref(t), ctypes.byref(by))
        names.append(name.value.decode())
    return names


def test_grid_barrier_wait_gives_up_and_handle_recovers(wp):
    """The persistent below-finest cycle (one cooperative launch whose phases meet at grid
    barriers): its last CTA skips the first barrier, every other CTA's wait runs out after 1 ms, the
    solve reports WP_ERR_DEVICE_WAIT, and the next solve on the handle matches the first one."""
    d, h, a, _, b = _sphere_case(wp, 64)
    mg = wp.CuMultigridFrac3D(*a, d, h)
    mg.SetTile(0, 3, 0, 1)  # the levels below the finest as one persistent launch
    opts = dict(rel_tol=1e-5, max_cycles=30, precision=wp.PREC_FP32, prolongation=wp.PROLONG_TRILINEAR)
    p0 = torch.zeros_like(b)
    box = {}
    names = _kernel_names(lambda: box.update(rep=mg.SolveTol(p0, None, b, **opts)))
    assert "mid_cycle" in names, names
    rep0 = box["rep"]
    assert rep0["status"] == "WP_OK", rep0
    wp.debug_withhold_wait(wp.WAIT_SITE_GRID_BARRIER, 0, 1e-3)
    p1 = torch.zeros_like(b)
    rep1 = mg.SolveTol(p1, None, b, raise_on_fail=False, **opts)
    assert rep1["status"] == "WP_ERR_DEVICE_WAIT", rep1
    assert "grid barrier" in wp._lib.last_error()
    p2 = torch.zeros_like(b)
    rep2 = mg.SolveTol(p2, None, b, **opts)
    assert rep2["status"] == "WP_OK" and rep2["cycles"] == rep0["cycles"], (rep0, rep2)
    assert torch.equal(p2, p0)


@pytest.mark.parametrize("at", [0, 5, 26])
def test_conv_pipeline_wait_gives_up_and_next_call_matches(wp, at):
    """Forward convolution: the first CTA does not load pipeline step `at`; its MMA thread's wait
    runs out after 1 ms, the loads already issued are drained and the tensor memory freed, the call
    raises WP_ERR_DEVICE_WAIT, and the next call gives the output of a call before it, bit for bit."""
    g = torch.Generator(device="cpu").manual_seed(11)
    x = torch.randn((4, 8, 16, 32), generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn((27, 32, 32), generator=g) / 30).to(torch.bfloat16).cuda()
    bias = torch.randn(32, generator=g).cuda()
    ref = torch.empty((4, 8, 16, 32), dtype=torch.bfloat16, device="cuda")
    wp.conv3_forward(ref, x, w, bias=bias)
    out = torch.zeros_like(ref)
    wp.debug_withhold_wait(wp.WAIT_SITE_CONV_PIPELINE, at, 1e-3)
    with pytest.raises(wp.WPError) as ei:
        wp.conv3_forward(out, x, w, bias=bias)
    assert ei.value.status == 7, str(ei.value)
    wp.conv3_forward(out, x, w, bias=bias)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


def test_conv_wgrad_wait_gives_up_and_next_call_matches(wp):
    g = torch.Generator(device="cpu").manual_seed(12)
    x = torch.randn((4, 8, 16, 16), generator=g).to(torch.bfloat16).cuda()
    gy = torch.randn((4, 8, 16, 32), generator=g).to(torch.bfloat16).cuda()
    ref = torch.zeros((27, 32, 16), device="cuda")
    wp.conv3_wgrad(ref, x, gy)
    dw = torch.zeros_like(ref)
    wp.debug_withhold_wait(wp.WAIT_SITE_CONV_PIPELINE, 0, 1e-3)
    with pytest.raises(wp.WPError) as ei:
        wp.conv3_wgrad(dw, x, gy)
    assert ei.value.status == 7, str(ei.value)
    dw.zero_()
    wp.conv3_wgrad(dw, x, gy)
    torch.cuda.synchronize()
    # FP32 atomics across CTAs: the sum order may differ from call to call
    assert torch.allclose(dw, ref, rtol=1e-5, atol=1e-5)


def test_withhold_is_one_shot_and_validated(wp):
    with pytest.raises(wp.WPError):
        wp.debug_withhold_wait(4, 0, 1e-3)
    with pytest.raises(wp.WPError):
        wp.debug_withhold_wait(wp.WAIT_SITE_CONV_PIPELINE, 0, 5.0)
    wp.debug_withhold_wait(wp.WAIT_SITE_CONV_PIPELINE, 0, 1e-3)
    wp.debug_withhold_wait(0, 0, 1e-3)  # disarmed: the next convolution runs normally
    x = torch.zeros((2, 4, 16, 16), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((27, 16, 16), dtype=torch.bfloat16, device="cuda")
    out = torch.empty((2, 4, 16, 16), dtype=torch.bfloat16, device="cuda")
    wp.conv3_forward(out, x, w)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_nonfinite_input_reports_nonfinite(wp, precision):
    """A NaN in the right-hand side: the solve reports WP_ERR_NONFINITE (the reference's solver has
    no such check; its iterate would silently fill with NaN) and the handle then solves a finite
    problem as before."""
    d, h, a, _, b = _sphere_case(wp, 32)
    prec = wp.PREC_FP32 if precision == "fp32" else wp.PREC_MIXED
    mg = wp.CuMultigridFrac3D(*a, d, h)
    opts = dict(rel_tol=1e-6, max_cycles=12, precision=prec)
    p0 = torch.zeros_like(b)
    rep0 = mg.SolveTol(p0, None, b, **opts)
    bad = b.clone()
    bad.view(-1)[bad.numel() // 3] = float("nan")
    p1 = torch.zeros_like(b)
    rep1 = mg.SolveTol(p1, None, bad, raise_on_fail=False, **opts)
    assert rep1["status"] == "WP_ERR_NONFINITE", rep1
    with pytest.raises(wp.WPError) as ei:
        mg.SolveTol(p1, None, bad, **opts)
    assert ei.value.status == 6
    p2 = torch.zeros_like(b)
    rep2 = mg.SolveTol(p2, None, b, **opts)
    assert rep2["status"] == "WP_OK" and rep2["cycles"] == rep0["cycles"]
    assert torch.allclose(p2, p0, rtol=0, atol=1e-6 * float(p0.abs().max()))


def test_projector_nonfinite_velocity(wp):
    d, h, a, u, _ = _sphere_case(wp, 32)
    pr = wp.Projector3D(*a, d, h, rel_tol=1e-8, max_cycles=40, autotune=False)
    s = wp.mac_shapes3d(*d)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    bad = [x.clone() for x in u]
    bad[1].view(-1)[17] = float("inf")
    rep = pr.run(*bad, *q)
    assert rep["status"] == "WP_ERR_NONFINITE", rep
    good = [x.clone() for x in u]
    rep = pr.run(*good, *q)
    assert rep["status"] == "WP_OK", rep
    assert torch.isfinite(q[0]).all() and rep["max_abs_div"] < 1e-2


def test_batch_replay_retests_the_tolerance_on_the_device(wp):
    """Each grid's solve in the batch graph is a device loop, so a replay runs as many steps as its
    input needs.  Grid 1 is planned on a zero field (no step needed) and replayed on a real one: it
    converges with steps of its own, the same count the single-grid path takes.  With the cycle cap
    below what the tolerance needs, both grids stop at the cap and wp_batch_results reports
    WP_ERR_NOT_CONVERGED with both flagged."""
    grids, u = [], []
    for i, n in enumerate((32, 64)):
        dd, h, a, ui, _ = _sphere_case(wp, n, seed=40 + i)
        grids.append({"dim": dd, "dx": h, "ax": a[0], "ay": a[1], "az": a[2]})
        u.append(ui)
    tol = 1e-9
    bp = wp.BatchProjector(grids, rel_tol=tol, max_cycles=40, nstreams=2)
    zero1 = [torch.zeros_like(x) for x in u[1]]
    cycles = bp.plan([u[0], zero1])
    assert cycles[0] >= 1 and cycles[1] == 0, cycles

    def outs():
        return [[torch.zeros(wp.mac_shapes3d(*g["dim"])[k], device="cuda") for k in ("qx", "qy", "qz")]
                for g in grids]

    bp.run([[x.clone() for x in u[0]], [x.clone() for x in zero1]], outs())
    res = bp.results()
    assert res["status"] == "WP_OK" and res["over_tol"] == [False, False], res
    assert res["cycles"] == cycles
    bp.run([[x.clone() for x in u[0]], [x.clone() for x in u[1]]], outs())
    res = bp.results()
    assert res["status"] == "WP_OK" and res["over_tol"] == [False, False], res
    assert res["rel_residual"][1] <= tol and res["cycles"][0] == cycles[0], res
    pr = wp.Projector3D(grids[1]["ax"], grids[1]["ay"], grids[1]["az"], grids[1]["dim"], grids[1]["dx"], rel_tol=tol,
                        max_cycles=40)
    q = [torch.zeros(wp.mac_shapes3d(*grids[1]["dim"])[k], device="cuda") for k in ("qx", "qy", "qz")]
    rep = pr.run(*[x.clone() for x in u[1]], *q)
    assert res["cycles"][1] == rep["cycles"] > 0, (res, rep)
    capped = wp.BatchProjector(grids, rel_tol=tol, max_cycles=2, nstreams=2)
    capped.run([[x.clone() for x in f] for f in u], outs())
    res = capped.results()
    assert res["status"] == "WP_ERR_NOT_CONVERGED" and res["over_tol"] == [True, True], res
    assert res["cycles"] == [2, 2], res