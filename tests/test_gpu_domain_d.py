"""Potential recovery with Dirichlet domain walls (bc 'd': cuProjectLocal_q_3d_nq_ccc between the
transforms with the boundary types swapped) through the C ABI, against the reference build's
fixtures and the FP64 oracle (relative L2 1e-5, the FP32 bound), and, at the benchmark sizes, the
size-independent property that it reproduces any discretely divergence-free field, wall flux
included: curl(recover(u)) == u."""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def N(t):
    return t.detach().double().cpu().numpy()


def rel(ref, got):
    ref, got = np.asarray(ref, np.float64), np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


@pytest.mark.parametrize("tag", ["p16x8x32", "p8", "r16", "r8x16x32"])
def test_domain_d_matches_reference_and_oracle(wp, oracle, tag):
    d = load_golden("domain_d")
    nx, ny, nz, h = d[tag + "_meta"]
    n = (int(nx), int(ny), int(nz))
    rec = wp.CuWaveletPotentialRecover3D(n, float(h), bc="d")
    s = wp.mac_shapes3d(*n)
    q = [torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")]  # every entry must be written
    u = [T(d[tag + "_" + k]) for k in ("xv", "yv", "zv")]
    u0 = [x.clone() for x in u]
    args = (d[tag + "_xv"], d[tag + "_yv"], d[tag + "_zv"], n, (float(h),) * 3)
    if tag[0] == "p":
        rec.ProjectLocal_q_ccc(*q, *u)
        oq = oracle.project3d(*args, bc="d")
    else:
        rec.Solve(*q, *u)
        oq = oracle.recover3d(*args, bc="d")
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(u, u0))  # inputs are read only
    for k, t, o in zip(("qx", "qy", "qz"), q, oq):
        assert rel(d[tag + "_" + k], N(t)) < 1e-5, (tag, k, rel(d[tag + "_" + k], N(t)))
        assert rel(o, N(t)) < 1e-5, (tag, k)


@pytest.mark.parametrize("n", [64, 256])
def test_domain_d_recovers_fields_with_wall_flux_at_full_size(wp, n):
    from waveletpotentials_b200 import fields
    rng = np.random.default_rng(n + 1)
    nn = (n, n, n)
    h = 1.0 / n
    s = wp.mac_shapes3d(*nn)
    q = [fields.spectral_field(s[k], -11.0 / 3.0, 1.0, rng) for k in ("qx", "qy", "qz")]
    u = fields.curl3d(*q, nn, (h, h, h))
    rec = wp.CuWaveletPotentialRecover3D(nn, h, bc="d")
    out = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    rec.Solve(*out, *(T(x) for x in u))
    c = fields.curl3d(*(N(t) for t in out), nn, (h, h, h))
    num = sum(np.sum((a - b) ** 2) for a, b in zip(u, c))
    den = sum(np.sum(a * a) for a in u)
    assert np.sqrt(num / den) < 1e-4


def test_domain_d_rejects_truncation(wp):
    rec = wp.CuWaveletPotentialRecover3D((8, 8, 8), 1.0 / 8, bc="d")
    s = wp.mac_shapes3d(8, 8, 8)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    with pytest.raises(wp.WPError):
        rec.CutCoefficients(*q, *q, 1)


@pytest.mark.parametrize("tag", ["p16", "p32x16", "p16x64", "p8x256", "r16", "r32x64", "r8x256"])
def test_domain_d2d_matches_reference_and_oracle(wp, oracle, tag):
    """2D: CuDivLocalProject::ProjectSingle with the Dirichlet-wall kernel (cuProjectLocal_q_single_n)
    and CuWaveletPotentialRecover2D::Solve with bc 'd', against the reference's FP32 build and the FP64
    oracle; every entry of qz is written and the inputs are left alone."""
    d = load_golden("domain_d2d")
    nx, ny, hx, hy = d[tag + "_meta"]
    n, h = (int(nx), int(ny)), (float(hx), float(hy))
    rec = wp.CuWaveletPotentialRecover2D(n, h, bc="d")
    qz = torch.full((n[0] + 1, n[1] + 1), 7.0, device="cuda")
    xv, yv = T(d[tag + "_xv"]), T(d[tag + "_yv"])
    x0, y0 = xv.clone(), yv.clone()
    args = (d[tag + "_xv"], d[tag + "_yv"], n, h)
    if tag[0] == "p":
        rec.ProjectSingle(qz, xv, yv)
        oq = oracle.project2d(*args, bc="d")
    else:
        rec.Solve(qz, xv, yv)
        oq = oracle.recover2d(*args, bc="d")
    torch.cuda.synchronize()
    assert torch.equal(xv, x0) and torch.equal(yv, y0)
    assert rel(d[tag + "_qz"], N(qz)) < 1e-5, (tag, rel(d[tag + "_qz"], N(qz)))
    assert rel(oq, N(qz)) < 1e-5, tag
