"""GPU parity: every CUDA entry point, called through the C ABI, against the reference's golden
fixtures and the FP64 oracle on the same seeded inputs.  Tolerances: FP32 kernels relative L2
<= 1e-5 against FP64 results (the north-star bound for velocity and potential); FP64 kernels 1e-12."""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def T(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def N(t):
    return t.detach().double().cpu().numpy()


def rel(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


@pytest.mark.parametrize("name", ["dwt1d", "dwt1d_cdf35", "dwt1d_families", "dwt1d_short"])
def test_dwt1d_fp32_and_fp64_match_reference(wp, name):
    d = load_golden(name)
    cases = [k[:-5] for k in d.files if k.endswith("_meta")]
    for b in cases:
        DX, DY, DZ, L, ax, bc, wav, fwd = (int(v) for v in d[b + "_meta"])
        ref = d[b + "_out"]
        for dt, tol in ((torch.float32, TOL32), (torch.float64, 1e-12)):
            src = T(d[b + "_in"], dt)
            dst = torch.empty_like(src)
            wp.CuWHHDForward.Solve1D(dst, src, (DX, DY, DZ), L, chr(ax), chr(bc), wav, bool(fwd))
            torch.cuda.synchronize()
            assert rel(ref, N(dst)) < tol, (b, dt, rel(ref, N(dst)))
            # in place gives the same result
            wp.CuWHHDForward.Solve1D(src, None, (DX, DY, DZ), L, chr(ax), chr(bc), wav, bool(fwd))
            assert torch.equal(src, dst), b


@pytest.mark.parametrize("wav,ext,bc", [(11, 0, "n"), (11, 0, "d"), (7, 1, "n"), (7, 1, "d"),
                                        (16, 1, "n"), (16, 1, "d"), (17, 0, "n"), (17, 0, "d"),
                                        (18, 0, "n"), (18, 0, "d")])
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_dwt_long_lines_against_oracle(wp, oracle, wav, ext, bc, axis):
    """Full 256(+1)-point lines along every axis (the 256^3 line length), both directions."""
    rng = np.random.default_rng(11)
    n = 256 + ext
    dims = {"x": (n, 40, 3), "y": (5, n, 3), "z": (3, 36, n)}[axis]
    a = rng.standard_normal((dims[2], dims[0], dims[1]))
    for fwd in (True, False):
        ref = oracle.dwt_axis(a, 8, axis, wav, bc, fwd)
        t = T(a)
        wp.CuWHHDForward.Solve1D(t, None, dims, 8, axis, bc, wav, fwd)
        assert rel(ref, N(t)) < TOL32


def test_ip_diag_matches_oracle_and_reference(wp, oracle):
    ip = load_golden("ip_tables")
    for k in ip.files:
        _, dim, wav, bc = k.split("_")
        g = wp.ip_diag(int(dim), int(wav), bc)
        np.testing.assert_allclose(g, oracle.ip_diag(int(dim), int(wav), bc), rtol=1e-12)
        np.testing.assert_allclose(g, ip[k][0], rtol=1e-6)


def test_project3d_matches_reference(wp):
    p = load_golden("project3d")
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    rec = wp.CuWaveletPotentialRecover3D(n, h)
    s = wp.mac_shapes3d(*n)
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]  # every entry must be written
    rec.ProjectLocal_q_ccc(*q, T(p["xv"]), T(p["yv"]), T(p["zv"]))
    for key, t in zip(("qx", "qy", "qz"), q):
        assert rel(p[key], N(t)) < TOL32, key


def test_project2d_matches_reference(wp):
    p = load_golden("project2d")
    n = tuple(int(v) for v in p["n"])
    rec = wp.CuWaveletPotentialRecover2D(n, float(p["h"]))
    qz = torch.full((n[0] + 1, n[1] + 1), 7.0, device="cuda")
    rec.ProjectSingle(qz, T(p["xv"]), T(p["yv"]))
    assert rel(p["qz"], N(qz)) < TOL32


@pytest.mark.parametrize("name", ["recover3d_16", "recover3d_aniso"])
def test_recover3d_matches_reference(wp, oracle, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    rec = wp.CuWaveletPotentialRecover3D(n, h)
    s = wp.mac_shapes3d(*n)
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]
    xv, yv, zv = T(p["xv"]), T(p["yv"]), T(p["zv"])
    xv0 = xv.clone()
    rec.Solve(*q, xv, yv, zv)
    assert torch.equal(xv, xv0)  # inputs are read only
    oq = oracle.recover3d(p["xv"], p["yv"], p["zv"], n, (h,) * 3)
    for key, t, o in zip(("qx", "qy", "qz"), q, oq):
        assert rel(p[key], N(t)) < TOL32, key
        assert rel(o, N(t)) < TOL32, key


@pytest.mark.parametrize("name", ["recover2d_32", "recover2d_aniso"])
def test_recover2d_matches_reference(wp, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    rec = wp.CuWaveletPotentialRecover2D(n, float(p["h"]))
    qz = torch.zeros((n[0] + 1, n[1] + 1), device="cuda")
    rec.Solve(qz, T(p["xv"]), T(p["yv"]))
    assert rel(p["qz"], N(qz)) < TOL32


@pytest.mark.parametrize("n", [128, 256])
def test_recover3d_reproduces_divergence_free_field_at_full_size(wp, n):
    """Size-independent property at the benchmark sizes: curl(recover(u)) == u for a discretely
    divergence-free u with zero wall-normal flux (the field-by-field comparison with the oracle at
    these sizes is in test_gpu_parity_fullsize.py)."""
    from waveletpotentials_b200 import fields
    rng = np.random.default_rng(n)
    nn = (n, n, n)
    h = 1.0 / n
    s = wp.mac_shapes3d(*nn)
    qx, qy, qz = (fields.spectral_field(s[k], -11.0 / 3.0, 1.0, rng) for k in ("qx", "qy", "qz"))
    qx[0] = qx[-1] = 0
    qx[:, :, 0] = qx[:, :, -1] = 0
    qy[0] = qy[-1] = 0
    qy[:, 0, :] = qy[:, -1, :] = 0
    qz[:, 0, :] = qz[:, -1, :] = 0
    qz[:, :, 0] = qz[:, :, -1] = 0
    xv, yv, zv = fields.curl3d(qx, qy, qz, nn, (h, h, h))
    rec = wp.CuWaveletPotentialRecover3D(nn, h)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    rec.Solve(*q, T(xv), T(yv), T(zv))
    ux, uy, uz = fields.curl3d(*(N(t) for t in q), nn, (h, h, h))
    num = sum(np.sum((a - b) ** 2) for a, b in zip((xv, yv, zv), (ux, uy, uz)))
    den = sum(np.sum(a * a) for a in (xv, yv, zv))
    assert np.sqrt(num / den) < 1e-4


def test_fractions_match_reference(wp):
    fr = load_golden("fractions3d")
    for n in (16, 32):
        sls = wp.CuSolidLevelSet3D((n, n, n), 1.0 / n)
        sls.InitLsSphere((0.5, 0.5, 0.5), float(fr[f"r_{n}"]))
        s = wp.mac_shapes3d(n, n, n)
        a = [torch.zeros(s[k], device="cuda") for k in ("xv", "yv", "zv")]
        sls.GetFrac(*a)
        for t, k in zip(a, ("ax", "ay", "az")):
            assert np.max(np.abs(N(t) - fr[f"{k}_{n}"])) < 1e-5


def test_divergence_gradient_and_max_match_reference(wp):
    p = load_golden("divgrad3d")
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    s = wp.mac_shapes3d(*n)
    b = torch.zeros(s["p"], device="cuda")
    args = [T(p[k]) for k in ("xv", "yv", "zv", "ax", "ay", "az")]
    wp.CuConvergence.GetB_3d_frac_vel(b, *args, n, h)
    assert rel(p["b"], N(b)) < TOL32
    assert abs(wp.max_abs(b) - np.max(np.abs(p["b"]))) <= 1e-5 * np.max(np.abs(p["b"]))
    xv, yv, zv = args[:3]
    wp.CuGradient.SubtractGradient3D_Frac_P(xv, yv, zv, T(p["p"]), *args[3:], n, h, True)
    for key, t in zip(("xv", "yv", "zv"), (xv, yv, zv)):
        assert rel(p[key + "_out"], N(t)) < TOL32


@pytest.mark.parametrize("name", ["mg3d_16", "mg3d_32"])
def test_mg3d_reference_cycles_match_reference(wp, name):
    """The reference V-cycle (constant prolongation) in FP32: per-cycle residual and solution."""
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    mg = wp.CuMultigridFrac3D(T(p["ax"]), T(p["ay"]), T(p["az"]), n, h)
    f = T(p["f"])
    dst = torch.zeros(f.shape, device="cuda")
    hist = []
    for c in range(int(p["ncycles"])):
        mg.Solve(dst, None if c == 0 else dst, f, 1, int(p["nu"][0]), int(p["nu"][1]), float(p["omega"]))
        hist.append(mg.GetResdualError(dst, f))
    # FP32 iterate against the FP64 reference: relative agreement plus an FP32 rounding floor
    assert np.all(np.abs(np.array(hist) - p["hist"]) <= 2e-3 * p["hist"] + 3e-6), (hist, p["hist"])
    assert rel(p["p"], N(dst)) < 1e-4


def test_mg2d_reference_cycles_match_reference(wp):
    p = load_golden("mg2d_32")
    n = tuple(int(v) for v in p["n"])
    mg = wp.CuMultigridFrac2D(T(p["ax"]), T(p["ay"]), n, float(p["h"]))
    f = T(p["f"])
    dst = torch.zeros(f.shape, device="cuda")
    mg.Solve(dst, None, f, int(p["ncycles"]), int(p["nu"][0]), int(p["nu"][1]), float(p["omega"]))
    assert rel(p["p"], N(dst)) < 1e-4
    assert abs(mg.GetResdualError(dst, f) / p["hist"][-1] - 1) < 1e-3


def active_cells(ax, ay, az):
    """Cells with a positive diagonal: at least one open interior face."""
    act = np.zeros((ax.shape[0], ay.shape[1], ax.shape[2]), dtype=bool)
    act[:, :-1, :] |= ax[:, 1:-1, :] > 0
    act[:, 1:, :] |= ax[:, 1:-1, :] > 0
    act[:, :, :-1] |= ay[:, :, 1:-1] > 0
    act[:, :, 1:] |= ay[:, :, 1:-1] > 0
    act[:-1] |= az[1:-1] > 0
    act[1:] |= az[1:-1] > 0
    return act


def _sphere_problem(wp, oracle, n, seed=0, spheres=None):
    from waveletpotentials_b200 import fields
    nn = (n, n, n)
    h = 1.0 / n
    c, r = ([[0.5, 0.5, 0.5]], [0.2]) if spheres is None else spheres
    sdf = oracle.sdf_spheres3d(nn, h, c, r)
    r32 = lambda a: a.astype(np.float32).astype(np.float64)  # both sides solve the FP32-stored problem
    ax, ay, az = (r32(a) for a in oracle.fractions3d(sdf, nn, h))
    xv, yv, zv = (r32(a) for a in fields.velocity3d(nn, seed))
    f = r32(oracle.divergence3d(xv, yv, zv, ax, ay, az, nn, (h,) * 3))
    return nn, h, (ax, ay, az), (xv, yv, zv), f


def test_mg3d_trilinear_matches_oracle_per_cycle(wp, oracle):
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32)
    _, ohist = oracle.mgfrac3d_solve(f, *a, nn, (h,) * 3, 8, 2, 2, 2 / 3, prolong=oracle.PROLONG_TRILINEAR)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, T(f), rel_tol=0.0, max_cycles=8, precision=wp.PREC_FP64)
    np.testing.assert_allclose(rep["history"], ohist, rtol=1e-6)


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-6), ("mixed", 1e-10), ("fp64", 1e-10)])
def test_mg3d_reaches_tolerance_checked_by_oracle(wp, oracle, precision, tol):
    nn, h, a, _, f = _sphere_problem(wp, oracle, 64, seed=3)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    dst = torch.zeros(f.shape, device="cuda")
    prec = {"fp32": wp.PREC_FP32, "mixed": wp.PREC_MIXED, "fp64": wp.PREC_FP64}[precision]
    rep = mg.SolveTol(dst, None, T(f), rel_tol=tol, max_cycles=60, precision=prec)
    assert rep["rel_residual"] <= tol
    # the solver removes the mean of f over the active cells (the operator's null space); check the
    # same compatible problem in FP64 with the oracle
    act = active_cells(*a)
    fc = f.copy()
    fc[act] -= f[act].mean()
    if precision == "fp32":
        sol = N(dst)
    else:
        sol = mg.Iterate64()  # the FP32 copy in dst is limited by FP32 storage
    _, r = oracle.frac_residual3d(sol, fc, *a, nn, (h,) * 3)
    orel = np.linalg.norm(r) / np.linalg.norm(f)
    assert orel <= tol * 1.5, (orel, rep)


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-6), ("mixed", 1e-10), ("fp64", 1e-10)])
def test_mg3d_fmg_start_checked_by_oracle(wp, oracle, precision, tol):
    """The full-multigrid start reaches the same tolerance (checked in FP64 by the oracle) in no more
    cycles than the zero start; both the batch-style fixed-cycle path and the one-grid path use it."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 64, seed=3)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    prec = {"fp32": wp.PREC_FP32, "mixed": wp.PREC_MIXED, "fp64": wp.PREC_FP64}[precision]
    dz = torch.zeros(f.shape, device="cuda")
    rz = mg.SolveTol(dz, None, T(f), rel_tol=tol, max_cycles=60, precision=prec)
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, T(f), rel_tol=tol, max_cycles=60, precision=prec, start=wp.START_FMG)
    assert rep["rel_residual"] <= tol and rep["cycles"] <= rz["cycles"], (rep["cycles"], rz["cycles"])
    assert rep["history"][0] < rz["history"][0]
    act = active_cells(*a)
    fc = f.copy()
    fc[act] -= f[act].mean()
    sol = N(dst) if precision == "fp32" else mg.Iterate64()
    _, r = oracle.frac_residual3d(sol, fc, *a, nn, (h,) * 3)
    assert np.linalg.norm(r) / np.linalg.norm(f) <= tol * 1.5


def test_mg_not_converged_is_reported(wp, oracle):
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    dst = torch.zeros(f.shape, device="cuda")
    rep = mg.SolveTol(dst, None, T(f), rel_tol=1e-12, max_cycles=2, precision=wp.PREC_MIXED, raise_on_fail=False)
    assert rep["status"] == "WP_ERR_NOT_CONVERGED" and rep["cycles"] == 2
    with pytest.raises(wp.WPError):
        mg.SolveTol(dst, None, T(f), rel_tol=1e-12, max_cycles=2, precision=wp.PREC_MIXED)


def test_projector_end_to_end(wp, oracle):
    nn, h, a, u, _ = _sphere_problem(wp, oracle, 32, seed=5)
    ta = [T(x) for x in a]
    proj = wp.Projector3D(*ta, nn, h, rel_tol=1e-10, precision=wp.PREC_MIXED)
    s = wp.mac_shapes3d(*nn)
    tu = [T(x) for x in u]
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    rep = proj.run(*tu, *q)
    assert rep["status"] == "WP_OK"
    # oracle: a (u - grad p) from the GPU pressure, and the recovered potential reproduces it
    pu = [N(t) for t in tu]
    b = oracle.divergence3d(*pu, *[np.ones_like(x) for x in pu], nn, (h,) * 3)
    assert abs(np.max(np.abs(b)) - rep["max_abs_div"]) <= 1e-2 * max(1.0, rep["max_abs_div"])
    oq = oracle.recover3d(*pu, nn, (h,) * 3)
    for o, t in zip(oq, q):
        assert rel(o, N(t)) < TOL32


def test_dst3d_matches_oracle(wp, oracle):
    n = (24, 20, 16)
    h = (1 / 25, 1 / 21, 1 / 17)
    rng = np.random.default_rng(21)
    f = rng.standard_normal((n[2], n[0], n[1]))
    ref = oracle.dst3d_poisson(f, n, h)
    dst = wp.CuDst3D(n, h)
    out = torch.zeros(f.shape, dtype=torch.float64, device="cuda")
    dst.Solve(out, T(f, torch.float64))
    assert rel(ref, N(out)) < 1e-12
    # in place
    g = T(f, torch.float64)
    dst.Solve(g, g)
    assert rel(ref, N(g)) < 1e-12


def test_boxes_and_2d_fractions_match_oracle(wp, oracle):
    n = (32, 24, 16)
    h = 1 / 32
    sls = wp.CuSolidLevelSet3D(n, h)
    sls.InitLsSpheres([[0.3, 0.3, 0.2]], [0.1])
    sls.AddBoxes([[0.5, 0.1, 0.1]], [[0.8, 0.4, 0.3]])
    ref = oracle.sdf_boxes3d(oracle.sdf_spheres3d(n, h, [[0.3, 0.3, 0.2]], [0.1]), n, h, [[0.5, 0.1, 0.1]],
                             [[0.8, 0.4, 0.3]])
    assert np.max(np.abs(N(sls.ls) - ref)) < 1e-6
    n2 = (40, 24)
    s2 = wp.CuSolidLevelSet2D(n2, 1 / 40)
    s2.InitLsCircles([[0.4, 0.3], [0.7, 0.5]], [0.12, 0.08])
    x = (np.arange(n2[0]) + 0.5) / 40
    y = (np.arange(n2[1]) + 0.5) / 40
    X, Y = np.meshgrid(x, y, indexing="ij")
    sdf = np.minimum(np.hypot(X - 0.4, Y - 0.3) - 0.12, np.hypot(X - 0.7, Y - 0.5) - 0.08)
    assert np.max(np.abs(N(s2.ls) - sdf)) < 1e-6
    ax = torch.zeros((n2[0] + 1, n2[1]), device="cuda")
    ay = torch.zeros((n2[0], n2[1] + 1), device="cuda")
    s2.GetFrac(ax, ay)
    oax, oay = oracle.fractions2d(sdf, n2, 1 / 40)
    assert np.max(np.abs(N(ax) - oax)) < 1e-5 and np.max(np.abs(N(ay) - oay)) < 1e-5


def test_recover2d_and_mg2d_full_config0_size(wp, oracle):
    """Config 0 size (256^2, no solids): 2D recovery against the oracle and a 2D tolerance solve."""
    from waveletpotentials_b200 import fields
    n = (256, 256)
    h = 1 / 256
    xv, yv = fields.velocity2d(n, 0)
    rec = wp.CuWaveletPotentialRecover2D(n, h)
    qz = torch.zeros((257, 257), device="cuda")
    rec.Solve(qz, T(xv), T(yv))
    ref = oracle.recover2d(xv.astype(np.float32), yv.astype(np.float32), n, (h, h))
    assert rel(ref, N(qz)) < TOL32
    ax, ay = np.ones((257, 256)), np.ones((256, 257))
    f = oracle.divergence2d(xv, yv, ax, ay, n, (h, h)).astype(np.float32).astype(np.float64)
    mg = wp.CuMultigridFrac2D(T(ax), T(ay), n, h)
    p = torch.zeros(n, device="cuda")
    rep = mg.SolveTol(p, None, T(f), rel_tol=1e-6, max_cycles=40, precision=wp.PREC_FP32)
    assert rep["rel_residual"] <= 1e-6


def test_mg_offset_views_and_autotune_keep_results(wp, oracle):
    """Right-hand sides that are 4-byte-offset views take the scalar column kernels, aligned ones the
    128-bit quad kernels (or the fused level-0 cycle), and the autotuner only reshapes grids: all
    give the same cycles, up to the constant that FP32 rounding adds to a Neumann iterate."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32, seed=9)
    mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
    fa = T(f)
    buf = torch.zeros(f.size + 1, device="cuda")
    buf[1:].copy_(fa.reshape(-1))
    fo = buf[1:].view(f.shape)  # contiguous, data pointer offset by 4 bytes
    assert fo.data_ptr() % 16 != 0
    outs = []
    for rhs in (fa, fo):
        dst = torch.zeros(f.shape, device="cuda")
        rep = mg.SolveTol(dst, None, rhs, rel_tol=0.0, max_cycles=6, precision=wp.PREC_FP32)
        outs.append((N(dst), rep["history"]))
    act = outs[0][0] != 0
    d = outs[0][0] - outs[1][0]
    d[act] -= d[act].mean()
    assert np.sqrt(np.sum(d * d) / np.sum(outs[0][0] ** 2)) < 1e-6
    np.testing.assert_allclose(outs[0][1], outs[1][1], rtol=1e-4)
    before = mg.Tiles()
    mg.Autotune()
    after = mg.Tiles()
    assert len(before) == len(after) and all(t[0] >= 1 for t in after)
    dst = torch.zeros(f.shape, device="cuda")
    dst0 = torch.zeros(f.shape, device="cuda")
    mg.Solve(dst, None, fa, n_iters=3, nu1=2, nu2=2, weight=2 / 3)
    mg2 = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)  # heuristic chunks
    mg2.Solve(dst0, None, fa, n_iters=3, nu1=2, nu2=2, weight=2 / 3)
    torch.cuda.synchronize()
    assert rel(N(dst0), N(dst)) < 1e-6


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6])
def test_mg_jacobi_variants_agree(wp, oracle, variant):
    """Register-budget variants, the fused two-sweep kernel and the TMA-staged sweep give the same
    cycles as the default one-sweep kernel (up to FP32 contraction order) for every pinned z-chunk."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32, seed=12)
    outs = []
    for var, zc in ((0, 0), (variant, 1), (variant, 5), (variant, 32)):
        mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
        for lvl in range(2):
            mg.SetTile(lvl, 0, zc, var)
        dst = torch.zeros(f.shape, device="cuda")
        rep = mg.SolveTol(dst, None, T(f), rel_tol=0.0, max_cycles=4, precision=wp.PREC_FP32)
        outs.append((N(dst), rep["history"]))
    for o in outs[1:]:
        assert rel(outs[0][0], o[0]) < 1e-6
        np.testing.assert_allclose(outs[0][1], o[1], rtol=1e-4)


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
def test_mg_restrict_variants_agree(wp, oracle, variant):
    """The register-budget variants of the fused residual-restriction give the default kernel's cycles."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32, seed=13)
    outs = []
    for var, zc in ((0, 0), (variant, 1), (variant, 3)):
        mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
        for lvl in range(2):
            mg.SetTile(lvl, 1, zc, var)
        dst = torch.zeros(f.shape, device="cuda")
        rep = mg.SolveTol(dst, None, T(f), rel_tol=0.0, max_cycles=4, precision=wp.PREC_FP32)
        outs.append((N(dst), rep["history"]))
    for o in outs[1:]:
        assert rel(outs[0][0], o[0]) < 1e-6
        np.testing.assert_allclose(outs[0][1], o[1], rtol=1e-4)


def test_mg_defect_variants_agree(wp, oracle):
    """The cp.async-pipelined FP64 defect gives the quad kernel's refinement history and iterate."""
    nn, h, a, _, f = _sphere_problem(wp, oracle, 32, seed=17)
    outs = []
    for var, zc in ((0, 0), (1, 2), (1, 32)):
        mg = wp.CuMultigridFrac3D(*(T(x) for x in a), nn, h)
        mg.SetTile(0, 2, zc, var)
        dst = torch.zeros(f.shape, device="cuda")
        rep = mg.SolveTol(dst, None, T(f), rel_tol=0.0, max_cycles=6, precision=wp.PREC_MIXED)
        outs.append((mg.Iterate64(), rep["history"]))
    for o in outs[1:]:
        assert rel(outs[0][0], o[0]) < 1e-12
        np.testing.assert_allclose(outs[0][1], o[1], rtol=1e-9)
