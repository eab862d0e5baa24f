"""Pins the FP64 oracle to the reference's own CUDA build (FP64): tests/golden/*.npz were produced
by tests/golden/make_golden.py through oracle/_ref/ref_driver on a B200."""
import numpy as np
import pytest

from conftest import load_golden


@pytest.mark.parametrize("name,count", [("dwt1d", 28), ("dwt1d_cdf35", 16), ("dwt1d_families", 72),
                                        ("dwt1d_short", 48)])
def test_dwt1d_matches_reference(oracle, name, count):
    d = load_golden(name)
    cases = [k[:-5] for k in d.files if k.endswith("_meta")]
    assert len(cases) >= count
    for b in cases:
        DX, DY, DZ, L, ax, bc, wav, fwd = (int(v) for v in d[b + "_meta"])
        out = oracle.dwt_axis(d[b + "_in"], L, chr(ax), wav, chr(bc), bool(fwd))
        ref = d[b + "_out"]
        err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
        assert err < 1e-12, (b, err)


def test_ip_tables_match_reference(oracle):
    ip = load_golden("ip_tables")
    for k in ip.files:
        _, dim, wav, bc = k.split("_")
        mine = oracle.ip_diag(int(dim), int(wav), bc)
        # the reference forms B B^T through a float tile and a float accumulator (cudaMath.cu:677-753)
        np.testing.assert_allclose(mine, ip[k][0], rtol=1e-6, err_msg=k)


@pytest.mark.parametrize("name", ["project3d"])
def test_project3d_matches_reference(oracle, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    qs = oracle.project3d(p["xv"], p["yv"], p["zv"], n, (h, h, h))
    for key, q in zip(("qx", "qy", "qz"), qs):
        assert oracle.rel_l2(p[key], q) < 1e-6, key


def test_project2d_matches_reference(oracle):
    p = load_golden("project2d")
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    assert oracle.rel_l2(p["qz"], oracle.project2d(p["xv"], p["yv"], n, (h, h))) < 1e-6


@pytest.mark.parametrize("name", ["recover3d_16", "recover3d_aniso"])
def test_recover3d_matches_reference(oracle, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    qs = oracle.recover3d(p["xv"], p["yv"], p["zv"], n, (h, h, h))
    for key, q in zip(("qx", "qy", "qz"), qs):
        assert oracle.rel_l2(p[key], q) < 1e-6, key


@pytest.mark.parametrize("name", ["recover2d_32", "recover2d_aniso"])
def test_recover2d_matches_reference(oracle, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    assert oracle.rel_l2(p["qz"], oracle.recover2d(p["xv"], p["yv"], n, (h, h))) < 1e-6


def test_fractions_match_reference(oracle):
    fr = load_golden("fractions3d")
    for n in (16, 32):
        r = float(fr[f"r_{n}"])
        sdf = oracle.sdf_spheres3d((n,) * 3, 1.0 / n, [[0.5, 0.5, 0.5]], [r])
        mine = oracle.fractions3d(sdf, (n,) * 3, 1.0 / n)
        for m, k in zip(mine, ("ax", "ay", "az")):
            # the reference takes sqrtf of the FP64 argument (cuSolidLevelSet3D.cu:32)
            assert np.max(np.abs(m - fr[f"{k}_{n}"])) < 1e-6


def test_divergence_and_gradient_match_reference(oracle):
    p = load_golden("divgrad3d")
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    b = oracle.divergence3d(p["xv"], p["yv"], p["zv"], p["ax"], p["ay"], p["az"], n, (h,) * 3)
    assert oracle.rel_l2(p["b"], b) < 1e-13
    u = oracle.grad_subtract3d(p["xv"], p["yv"], p["zv"], p["p"], p["ax"], p["ay"], p["az"], n, (h,) * 3, True)
    for key, m in zip(("xv", "yv", "zv"), u):
        assert oracle.rel_l2(p[key + "_out"], m) < 1e-13


@pytest.mark.parametrize("name", ["mg3d_16", "mg3d_32"])
def test_mg3d_matches_reference_per_cycle(oracle, name):
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    sol, hist = oracle.mgfrac3d_solve(p["f"], p["ax"], p["ay"], p["az"], n, (h,) * 3, int(p["ncycles"]),
                                      int(p["nu"][0]), int(p["nu"][1]), float(p["omega"]))
    np.testing.assert_allclose(hist, p["hist"], rtol=1e-9)
    assert oracle.rel_l2(p["p"], sol) < 1e-11


@pytest.mark.parametrize("name", ["mg3d_index_pores", "mg3d_index_island", "mg3d_index_sphere32"])
def test_mg3d_index_matches_reference_per_cycle(oracle, name):
    """CuMultigridFrac3D::Solve_index, one cycle per call: the oracle's index-sparse cycle, including
    the residual workspace shared by the levels and nu1 post-sweeps, follows the reference build."""
    p = load_golden(name)
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    sol, hist, counts = oracle.mgfrac3d_solve_index(p["f"], p["ax"], p["ay"], p["az"], n, (h,) * 3,
                                                    int(p["ncycles"]), int(p["nu"][0]), int(p["nu"][1]),
                                                    float(p["omega"]))
    np.testing.assert_allclose(hist, p["hist"], rtol=1e-9)
    assert oracle.rel_l2(p["p"], sol) < 1e-11
    assert counts[0] < np.prod(n) and (name != "mg3d_index_island" or counts[1] == 0)


def test_mg3d_index_oracle_reduces_to_the_dense_cycle_without_solids(oracle):
    """Every cell listed: the index-sparse cycle is the reference V-cycle with nu2 = nu1."""
    n = (12, 10, 8)
    s = oracle.mac_shapes3d(*n)
    rng = np.random.default_rng(4)
    a = [np.ones(s[k]) for k in ("xv", "yv", "zv")]
    f = rng.standard_normal(s["p"])
    pi, hi, counts = oracle.mgfrac3d_solve_index(f, *a, n, (0.1,) * 3, 3, 2, 5, 0.8)
    pd, hd = oracle.mgfrac3d_solve(f, *a, n, (0.1,) * 3, 3, 2, 2, 0.8)
    assert list(counts) == [int(np.prod(n)), 6 * 5 * 4, 3 * 3 * 2]
    np.testing.assert_allclose(hi, hd, rtol=1e-13)
    assert oracle.rel_l2(pd, pi) < 1e-13


def test_cut3d_matches_reference(oracle):
    """CuWaveletPotentialRecover3D::CutCoefficients at every level, two shapes."""
    g = load_golden("cut3d")
    for key in [k for k in g.files if k.startswith("n_")]:
        tag = key[2:]
        n = tuple(int(v) for v in g[key])
        q = [g[f"{k}_{tag}"] for k in ("qx", "qy", "qz")]
        for level in range(int(np.log2(min(n))) + 1):
            out = oracle.cut3d(*q, n, level)
            for k, o, a in zip(("qx", "qy", "qz"), out, q):
                # against the input: the deepest cut leaves rounding noise only
                d = np.linalg.norm(o - g[f"{k}_{tag}_cut{level}"]) / np.linalg.norm(a)
                assert d < 1e-12, (tag, level, k, d)
            if level == 0:
                assert all(oracle.rel_l2(a, o) < 1e-13 for a, o in zip(q, out))


def test_subsampled_fractions_match_reference(oracle):
    """The static CuSolidLevelSet3D::GetFrac: open / closed by the quadratic interpolant at the face
    centre, cut faces as a count of 128 x 128 trilinear samples (up to a few samples that lie within
    rounding of the zero level)."""
    g = load_golden("frac3d_sub")
    for key in [k for k in g.files if k.startswith("n_")]:
        tag = key[2:]
        n = tuple(int(v) for v in g[key])
        out = oracle.fractions3d_subsampled(g[f"ls_{tag}"], n, 1.0 / n[0])
        for k, o in zip(("ax", "ay", "az"), out):
            d = np.abs(o - g[f"{k}_{tag}"])
            assert d.max() <= 3.0 / 16384 and np.count_nonzero(d) <= 3, (tag, k, d.max(), np.count_nonzero(d))


def test_fast_sweep_matches_reference_fixed_point(oracle):
    """CuFastSweeping::ReinitLevelSet and Solve, past convergence: the oracle's Jacobi iterations
    reach the reference's fixed point."""
    g = load_golden("fsweep")
    n = tuple(int(v) for v in g["n"])
    for mode, reinit in (("reinit", True), ("solve", False)):
        out = oracle.fast_sweep(g["ls_" + mode], n, float(g["h"]), int(g["iters"]), reinit)
        ref = g["out_" + mode]
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), (mode, np.abs(out - ref).max())
    out = oracle.particles_to_ls(g["particles"], n, float(g["h"]), float(g["radius"]), float(g["max_dis"]),
                                 int(g["iters"]))
    ref = g["out_particles"]
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), np.abs(out - ref).max()


@pytest.mark.parametrize("start", ["band", "wavy"])
def test_particles_to_ls_narrow_matches_reference_fixed_point(oracle, start):
    """CuFastSweeping::ParticlesToLsNarrow from a constant band and from a wavy level set, past
    convergence: the oracle reaches the reference's fixed point."""
    g = load_golden("p2ls_narrow")
    n = tuple(int(v) for v in g["n"])
    out = oracle.particles_to_ls_narrow(g[start + "_ls"], g[start + "_particles"], n, float(g["h"]),
                                        float(g["radius"]), int(g["iters"]))
    ref = g[start + "_out"]
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max(), np.abs(out - ref).max()


def test_mg2d_matches_reference_per_cycle(oracle):
    p = load_golden("mg2d_32")
    n = tuple(int(v) for v in p["n"])
    h = float(p["h"])
    sol, hist = oracle.mgfrac2d_solve(p["f"], p["ax"], p["ay"], n, (h,) * 2, int(p["ncycles"]), int(p["nu"][0]),
                                      int(p["nu"][1]), float(p["omega"]))
    np.testing.assert_allclose(hist, p["hist"], rtol=1e-9)
    assert oracle.rel_l2(p["p"], sol) < 1e-11


@pytest.mark.parametrize("tag", ["15", "8"])
def test_dst3d_matches_reference(oracle, tag):
    """CuDst3D::Solve (cuDst3D.cu:265-341) of the reference build: the oracle's exact DST-I agrees
    to the FP32 rounding of the reference's transform constants (it forms sqrt(2/(n+1)) and
    1/(n+1) in single precision even in its FP64 build, cuDst3D.cu:267-269, 314)."""
    g = load_golden("dst3d")
    f, p, d = g["f_" + tag], g["p_" + tag], tuple(float(v) for v in g["d_" + tag])
    n = f.shape[0]
    got = oracle.dst3d_poisson(f, (n, n, n), d)
    assert np.linalg.norm(got - p) <= 2e-7 * np.linalg.norm(p)


@pytest.mark.parametrize("n", [8, 16])
def test_sweep_recovery_matches_reference(oracle, n):
    """CuParallelSweep3D with bc 'n' of the reference build (cuParallelSweep3D.cu:939-966 Solve,
    :1043-1081 ProjectZero): the line sweeps agree exactly; the projection (a DST-I Poisson solve on
    the (n-1)^3 interior nodes) agrees to the FP32 rounding of the reference's DST constants, which
    vanishes at n = 8 where sqrt(2/(n-1+1)) = 1/2 is exact in single precision."""
    g = load_golden("psweep")
    h = 1.0 / n
    nn, d = (n, n, n), (h, h, h)
    u = [g[f"{k}_{n}"] for k in ("xv", "yv", "zv")]
    qs = oracle.sweep3d_solve(*u, nn, d)
    for a, k in zip(qs, ("qx", "qy", "qz")):
        ref = g[f"{k}_solve_{n}"]
        assert np.abs(a - ref).max() <= 1e-14 * np.abs(ref).max()
    qp = oracle.sweep3d_project(*qs, nn, d)
    tol = 1e-13 if n == 8 else 1e-6
    for a, k in zip(qp, ("qx", "qy", "qz")):
        ref = g[f"{k}_{n}"]
        assert np.abs(a - ref).max() <= tol * np.abs(ref).max()


def test_sweep2d_matches_reference(oracle):
    """CuParallelSweep3D(int2, DTYPE2, 'n')::Solve(qz, xv, yv) (cuParallelSweep3D.cu:987-1000)."""
    g = load_golden("psweep")
    n = 32
    qz = oracle.sweep2d_solve(g["yv2d"], (n, n), (1.0 / n, 1.0 / n))
    assert np.abs(qz - g["qz2d"]).max() <= 1e-14 * np.abs(g["qz2d"]).max()


@pytest.mark.parametrize("n", [8, 16])
def test_sweep_solve_with_dirichlet_walls_matches_reference(oracle, n):
    """CuParallelSweep3D::Solve with bc 'd' (qy's z = 0 plane from the x-integral of zv's bottom face,
    no top-plane step) on a field with wall flux, and the 2D Solve with bc 'd': exact sequential sums."""
    g = load_golden("psweep_d")
    h = 1.0 / n
    qs = oracle.sweep3d_solve(*[g[f"{k}_{n}"] for k in ("xv", "yv", "zv")], (n, n, n), (h, h, h), bc="d")
    for a, k in zip(qs, ("qx", "qy", "qz")):
        ref = g[f"{k}_solve_{n}"]
        assert np.abs(a - ref).max() <= 1e-14 * max(np.abs(ref).max(), 1e-300), k
    qz = oracle.sweep2d_solve(g["yv2d"], (32, 32), (1 / 32, 1 / 32), bc="d", xv=g["xv2d"])
    assert np.abs(qz - g["qz2d"]).max() <= 1e-14 * np.abs(g["qz2d"]).max()


@pytest.mark.parametrize("tag", ["a8", "b16", "c8"])
def test_sweep_solve_from_mid_matches_reference(oracle, tag):
    """CuParallelSweep3D::SolveFromMid from interior and zero mid indices: exact sequential sums."""
    g = load_golden("psweep_mid")
    n, mx, my, mz = (int(v) for v in g[tag + "_meta"])
    h = 1.0 / n
    q = oracle.sweep3d_solve_from_mid(*[g[f"{tag}_{k}"] for k in ("xv", "yv", "zv")], (n, n, n), (h, h, h),
                                      (mx, my, mz))
    for a, k in zip(q, ("qx", "qy", "qz")):
        ref = g[f"{tag}_{k}"]
        assert np.abs(a - ref).max() <= 1e-14 * max(np.abs(ref).max(), 1.0), k


@pytest.mark.parametrize("tag", ["p16x8x32", "p8", "r16", "r8x16x32"])
def test_domain_d_projection_and_recovery_match_reference(oracle, tag):
    """Dirichlet domain walls: CuDivLocalProject3D::ProjectLocal_q_ccc with bc_base 'n'
    (cuProjectLocal_q_3d_nq_ccc, the wall planes, lines and corner included) on random coefficients
    ("p" cases) and CuWaveletPotentialRecover3D::Solve with bc 'd' on random fields with wall flux
    ("r" cases), from the reference's FP64 build.  The reference's inner-product tables carry FP32
    rounding, hence the 1e-7."""
    d = load_golden("domain_d")
    nx, ny, nz, h = d[tag + "_meta"]
    n = (int(nx), int(ny), int(nz))
    args = (d[tag + "_xv"], d[tag + "_yv"], d[tag + "_zv"], n, (h,) * 3)
    q = oracle.project3d(*args, bc="d") if tag[0] == "p" else oracle.recover3d(*args, bc="d")
    for k, got in zip(("qx", "qy", "qz"), q):
        ref = d[tag + "_" + k]
        assert np.sqrt(np.sum((ref - got) ** 2) / np.sum(ref * ref)) < 1e-7, (tag, k)


@pytest.mark.parametrize("tag", ["p16", "p32x16", "p16x64", "p8x256", "r16", "r32x64", "r8x256"])
def test_domain_d2d_projection_and_recovery_match_reference(oracle, tag):
    """2D Dirichlet domain walls: CuDivLocalProject::ProjectSingle with bc_base 'n'
    (cuProjectLocal_q_single_n: its wall rows' 2 x 2 solves and the GetDivL0Matrix corner, for axes
    0, 1, 2 and 5 levels apart) on random coefficients ("p" cases) and CuWaveletPotentialRecover2D::Solve
    with bc 'd' on random fields with wall flux ("r" cases).  From the reference's FP32 build (its FP64
    build cannot launch this kernel: 72 registers a thread in 1024-thread blocks), hence the 3e-6."""
    d = load_golden("domain_d2d")
    nx, ny, hx, hy = d[tag + "_meta"]
    n, h = (int(nx), int(ny)), (float(hx), float(hy))
    args = (d[tag + "_xv"], d[tag + "_yv"], n, h)
    got = oracle.project2d(*args, bc="d") if tag[0] == "p" else oracle.recover2d(*args, bc="d")
    ref = d[tag + "_qz"]
    assert np.sqrt(np.sum((ref - got) ** 2) / np.sum(ref * ref)) < 3e-6, tag
    assert np.max(np.abs(ref - got)) < 1e-6 * max(1.0, np.max(np.abs(ref))), tag
