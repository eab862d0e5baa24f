"""Tensor-core 3x3x3 convolutions (tcgen05, BF16 operands, FP32 accumulation) against the FP64
oracle on the same BF16-rounded inputs.  Forward and input-gradient outputs are stored in BF16
(tolerance 5e-3 relative L2, about two BF16 ulps); the weight gradient is FP32 (1e-4)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


def B(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda").to(torch.bfloat16)


def F(t):
    return t.float().cpu().numpy().astype(np.float64)


SHAPES = [(8, 16, 16), (2, 2, 128), (3, 4, 8), (2, 8, 256)]


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 16), (32, 64), (64, 64), (64, 32)])
def test_conv3_forward_matches_oracle(wp, oracle, cin, cout):
    rng = np.random.default_rng(cin * 100 + cout)
    for nz, nx, ny in SHAPES:
        x = oracle.bf16_round(rng.standard_normal((nz, nx, ny, cin)))
        w = oracle.bf16_round(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
        b = rng.standard_normal(cout).astype(np.float32)
        ref = oracle.conv3d_forward(x, w, b)
        out = torch.empty((nz, nx, ny, cout), dtype=torch.bfloat16, device="cuda")
        wp.conv3_forward(out, B(x), B(w), bias=torch.as_tensor(b, device="cuda"))
        torch.cuda.synchronize()
        assert rel(ref, F(out)) < 5e-3, (nz, nx, ny, rel(ref, F(out)))
        wp.conv3_forward(out, B(x), B(w), bias=torch.as_tensor(b, device="cuda"), relu=True)
        assert rel(np.maximum(ref, 0), F(out)) < 5e-3


def test_conv3_two_parts_addend_mask(wp, oracle):
    rng = np.random.default_rng(7)
    nz, nx, ny = 4, 8, 16
    x0 = oracle.bf16_round(rng.standard_normal((nz, nx, ny, 32)))
    x1 = oracle.bf16_round(rng.standard_normal((nz, nx, ny, 64)))
    w0 = oracle.bf16_round(rng.standard_normal((27, 32, 32)) * 0.05)
    w1 = oracle.bf16_round(rng.standard_normal((27, 32, 64)) * 0.05)
    ad = oracle.bf16_round(rng.standard_normal((nz, nx, ny, 32)))
    mk = oracle.bf16_round(rng.standard_normal((nz, nx, ny, 32)))
    ref = oracle.conv3d_forward(x0, w0) + oracle.conv3d_forward(x1, w1) + ad
    ref = np.where(mk > 0, ref, 0.0)
    out = torch.empty((nz, nx, ny, 32), dtype=torch.bfloat16, device="cuda")
    wp.conv3_forward(out, B(x0), B(w0), x1=B(x1), w1=B(w1), addend=B(ad), mask=B(mk))
    torch.cuda.synchronize()
    assert rel(ref, F(out)) < 5e-3


@pytest.mark.parametrize("cin,cout", [(16, 16), (32, 64), (64, 32)])
def test_conv3_input_grad_via_flipped_weights(wp, oracle, cin, cout):
    rng = np.random.default_rng(3)
    nz, nx, ny = 4, 8, 32
    gy = oracle.bf16_round(rng.standard_normal((nz, nx, ny, cout)))
    w = oracle.bf16_round(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cout))
    ref = oracle.conv3d_input_grad(gy, w)
    wt = np.ascontiguousarray(np.transpose(w[::-1], (0, 2, 1)))
    out = torch.empty((nz, nx, ny, cin), dtype=torch.bfloat16, device="cuda")
    wp.conv3_forward(out, B(gy), B(wt))
    torch.cuda.synchronize()
    assert rel(ref, F(out)) < 5e-3


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 64), (32, 32), (64, 16), (64, 64)])
def test_conv3_weight_grad_matches_oracle(wp, oracle, cin, cout):
    rng = np.random.default_rng(cin + cout)
    for nz, nx, ny in [(4, 8, 16), (2, 2, 128)]:
        x = oracle.bf16_round(rng.standard_normal((nz, nx, ny, cin)))
        gy = oracle.bf16_round(rng.standard_normal((nz, nx, ny, cout)))
        ref = oracle.conv3d_weight_grad(x, gy)
        dw = torch.zeros((27, cout, cin), dtype=torch.float32, device="cuda")
        wp.conv3_wgrad(dw, B(x), B(gy))
        torch.cuda.synchronize()
        assert rel(ref, dw.cpu().numpy()) < 1e-4, (nz, nx, ny, rel(ref, dw.cpu().numpy()))


def test_conv3_rejects_bad_channels(wp):
    x = torch.zeros((2, 4, 4, 8), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((27, 16, 8), dtype=torch.bfloat16, device="cuda")
    out = torch.zeros((2, 4, 4, 16), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(wp.WPError):
        wp.conv3_forward(out, x, w)
