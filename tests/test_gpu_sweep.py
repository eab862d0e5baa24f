"""Sweep + DST potential recovery (CuParallelSweep3D) against the FP64 oracle."""
import numpy as np
import pytest
import torch

from test_oracle_properties import _wall_compatible_potential

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float32), device="cuda")


def _rel(ref, got):
    return float(np.abs(np.asarray(got, np.float64) - ref).max() / max(np.abs(ref).max(), 1e-300))


@pytest.mark.parametrize("n", [(32, 32, 32), (24, 16, 20), (7, 9, 5)])
def test_sweep_solve_and_project_match_oracle(wp, oracle, n):
    d = (1.0 / 32,) * 3
    s = oracle.mac_shapes3d(*n)
    u = [a.astype(np.float32).astype(np.float64) for a in oracle.curl3d(*_wall_compatible_potential(s, 5), n, d)]
    sw = wp.CuParallelSweep3D(n, d, "n")
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]  # Solve overwrites every entry
    sw.Solve(*q, *(_t(a) for a in u))
    torch.cuda.synchronize()
    ref = oracle.sweep3d_solve(*u, n, d)
    for r, g in zip(ref, q):
        assert _rel(r, g.cpu().numpy()) < 2e-6
    # projection of the same (FP32-stored) potential on both sides
    q32 = [a.astype(np.float32).astype(np.float64) for a in ref]
    qg = [_t(a) for a in q32]
    sw.Project(*qg)
    torch.cuda.synchronize()
    refp = oracle.sweep3d_project(*q32, n, d)
    for r, g in zip(refp, qg):
        assert _rel(r, g.cpu().numpy()) < 2e-5


def test_sweep_recovers_curl_at_128(wp, oracle):
    """curl q = u after Solve + Project on a 128^3 divergence-free field with no normal flux."""
    n = (128, 128, 128)
    d = (1.0 / 128,) * 3
    s = oracle.mac_shapes3d(*n)
    u = [a.astype(np.float32).astype(np.float64) for a in oracle.curl3d(*_wall_compatible_potential(s, 9), n, d)]
    sw = wp.CuParallelSweep3D(n, d, "n")
    q = [torch.empty(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    sw.Solve(*q, *(_t(a) for a in u))
    sw.Project(*q)
    torch.cuda.synchronize()
    got = oracle.curl3d(*(t.cpu().numpy().astype(np.float64) for t in q), n, d)
    assert oracle.rel_l2_multi(u, got) < 1e-5
    nx, ny, nz = n
    px, py, pz = (t.cpu().numpy().astype(np.float64) for t in q)
    div = ((px[1:nz, 1:nx, 1:ny] - px[1:nz, 0:nx - 1, 1:ny]) + (py[1:nz, 1:nx, 1:ny] - py[1:nz, 1:nx, 0:ny - 1]) +
           (pz[1:nz, 1:nx, 1:ny] - pz[0:nz - 1, 1:nx, 1:ny])) / d[0]
    assert np.abs(div).max() <= 1e-3 * np.abs(px).max() / d[0]


@pytest.mark.parametrize("n", [(32, 48), (257, 33)])
def test_sweep2d_matches_oracle(wp, oracle, n):
    d = (1.0 / 64, 1.0 / 64)
    rng = np.random.default_rng(2)
    yv = rng.standard_normal((n[0], n[1] + 1)).astype(np.float32).astype(np.float64)
    xv = np.zeros((n[0] + 1, n[1]))
    qz = torch.full((n[0] + 1, n[1] + 1), 3.0, device="cuda")
    wp.CuParallelSweep3D.Solve2D(qz, _t(xv), _t(yv), n, d[0], "n")
    torch.cuda.synchronize()
    assert _rel(oracle.sweep2d_solve(yv, n, d), qz.cpu().numpy()) < 2e-6


def test_sweep_rejects_other_boundaries(wp):
    with pytest.raises(wp.WPError):
        wp.CuParallelSweep3D((8, 8, 8), 1.0 / 8, "z")
    qz = torch.zeros((9, 9), device="cuda")
    yv = torch.zeros(wp.mac_shapes2d(8, 8)["yv"], device="cuda")
    with pytest.raises(wp.WPError):
        wp.CuParallelSweep3D.Solve2D(qz, None, yv, (8, 8), 1.0 / 8, bc="d")  # bc 'd' reads xv


@pytest.mark.parametrize("tag", ["15", "8"])
def test_dst3d_matches_reference(wp, tag):
    """The GPU's DST-I solve (handle and allocation-free entry points, FP64) against the reference
    build's CuDst3D::Solve: within the FP32 rounding of the reference's transform constants."""
    from conftest import load_golden
    g = load_golden("dst3d")
    f, p, d = g["f_" + tag], g["p_" + tag], tuple(float(v) for v in g["d_" + tag])
    n = f.shape[0]
    tf = torch.as_tensor(f, dtype=torch.float64, device="cuda")
    out = torch.empty_like(tf)
    dst = wp.CuDst3D((n, n, n), d)
    dst.Solve(out, tf)
    out2 = torch.empty_like(tf)
    wp.CuDst3D.SolveNoAlloc(out2, tf, (n, n, n), d)
    torch.cuda.synchronize()
    for got in (out, out2):
        g64 = got.cpu().numpy()
        assert np.linalg.norm(g64 - p) <= 2e-7 * np.linalg.norm(p)
    dst.close()


@pytest.mark.parametrize("n", [8, 16])
def test_sweep_recovery_matches_reference(wp, n):
    """The GPU's sweep + DST recovery (FP32 sweeps, FP64 DST) against the reference build's
    CuParallelSweep3D Solve and Project on the same divergence-free field (within FP32 rounding of
    the line integrals and, at 16^3, the reference's single-precision DST constants)."""
    from conftest import load_golden
    g = load_golden("psweep")
    h = 1.0 / n
    u = [_t(g[f"{k}_{n}"]) for k in ("xv", "yv", "zv")]
    s = wp.mac_shapes3d(n, n, n)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    sw = wp.CuParallelSweep3D((n, n, n), h, "n")
    sw.Solve(*q, *u)
    torch.cuda.synchronize()
    for t, k in zip(q, ("qx", "qy", "qz")):
        assert _rel(g[f"{k}_solve_{n}"], t.cpu().numpy()) < 2e-6
    sw.Project(*q)
    torch.cuda.synchronize()
    for t, k in zip(q, ("qx", "qy", "qz")):
        assert _rel(g[f"{k}_{n}"], t.cpu().numpy()) < 1e-5
    sw.close()


def test_sweep2d_matches_reference(wp):
    """CuParallelSweep3D(int2, DTYPE2, 'n')::Solve(qz, xv, yv) of the reference build."""
    from conftest import load_golden
    g = load_golden("psweep")
    n = 32
    qz = torch.zeros((n + 1, n + 1), device="cuda")
    wp.CuParallelSweep3D.Solve2D(qz, _t(g["xv2d"]), _t(g["yv2d"]), (n, n), 1.0 / n)
    torch.cuda.synchronize()
    assert _rel(g["qz2d"], qz.cpu().numpy()) < 2e-6


@pytest.mark.parametrize("n", [8, 16])
def test_sweep_solve_with_dirichlet_walls_matches_reference(wp, n):
    """bc 'd': CuParallelSweep3D::Solve (qy's z = 0 plane from zv's bottom face) and the 2D Solve
    against the reference build; Project, the reference's ProjectD, is refused (not built)."""
    from conftest import load_golden
    g = load_golden("psweep_d")
    h = 1.0 / n
    u = [_t(g[f"{k}_{n}"]) for k in ("xv", "yv", "zv")]
    s = wp.mac_shapes3d(n, n, n)
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]
    sw = wp.CuParallelSweep3D((n, n, n), h, "d")
    sw.Solve(*q, *u)
    torch.cuda.synchronize()
    for t, k in zip(q, ("qx", "qy", "qz")):
        assert _rel(g[f"{k}_solve_{n}"], t.cpu().numpy()) < 2e-6, k
    with pytest.raises(wp.WPError):
        sw.Project(*q)
    sw.close()
    qz = torch.full((33, 33), 7.0, device="cuda")
    wp.CuParallelSweep3D.Solve2D(qz, _t(g["xv2d"]), _t(g["yv2d"]), (32, 32), 1.0 / 32, bc="d")
    torch.cuda.synchronize()
    assert _rel(g["qz2d"], qz.cpu().numpy()) < 2e-6


@pytest.mark.parametrize("tag", ["a8", "b16", "c8"])
def test_sweep_solve_from_mid_matches_reference(wp, tag):
    """CuParallelSweep3D::SolveFromMid (both-way integrals from a mid plane and row) against the
    reference build, every entry written; a mid index outside the grid is refused."""
    from conftest import load_golden
    g = load_golden("psweep_mid")
    n, mx, my, mz = (int(v) for v in g[tag + "_meta"])
    h = 1.0 / n
    u = [_t(g[f"{tag}_{k}"]) for k in ("xv", "yv", "zv")]
    s = wp.mac_shapes3d(n, n, n)
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]
    sw = wp.CuParallelSweep3D((n, n, n), h, "n")
    sw.SolveFromMid(*q, *u, (mx, my, mz))
    torch.cuda.synchronize()
    for t, k in zip(q, ("qx", "qy", "qz")):
        ref = g[f"{tag}_{k}"]
        got = t.cpu().numpy()
        if np.abs(ref).max() == 0:
            assert np.abs(got).max() == 0, k
        else:
            assert _rel(ref, got) < 2e-6, (k, _rel(ref, got))
    with pytest.raises(wp.WPError):
        sw.SolveFromMid(*q, *u, (n + 1, 0, 0))
    sw.close()


def test_dirichlet_sweep_and_mid_sweep_reproduce_fields_at_64(wp):
    """At 64^3, FP32: curl q = u after the bc 'd' solve and after SolveFromMid, for a field with wall flux."""
    from waveletpotentials_b200 import fields
    n = 64
    h = 1.0 / n
    rng = np.random.default_rng(5)
    s = wp.mac_shapes3d(n, n, n)
    q0 = [fields.spectral_field(s[k], -11.0 / 3.0, 1.0, rng) for k in ("qx", "qy", "qz")]
    u = fields.curl3d(*q0, (n, n, n), (h, h, h))
    den = sum(np.sum(a * a) for a in u)
    for bc, mid in (("d", None), ("n", (20, 0, 41))):
        sw = wp.CuParallelSweep3D((n, n, n), h, bc)
        q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
        if mid is None:
            sw.Solve(*q, *[_t(a) for a in u])
        else:
            sw.SolveFromMid(*q, *[_t(a) for a in u], mid)
        torch.cuda.synchronize()
        c = fields.curl3d(*[t.double().cpu().numpy() for t in q], (n, n, n), (h, h, h))
        assert np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(u, c)) / den) < 1e-5, (bc, mid)
        sw.close()
