"""Warm-start network: its GPU forward, loss and gradients (tensor-core convolutions, BF16
activations) against the FP64 oracle network; the device field generator; and what training buys
the multigrid (V-cycles to the same tolerance, with the zero-start fallback)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def _groups(oracle):
    """Slices of the flat parameter vector: one per convolution (weights + bias) and the head."""
    out, off = [], 0
    for cin0, cin1, cout in oracle.UNET_SPEC:
        n = 27 * cout * (cin0 + cin1) + cout
        out.append(slice(off, off + n))
        off += n
    out.append(slice(off, off + 17))
    return out


def test_unet_forward_and_gradients_match_oracle(wp, oracle):
    nx, ny, nz = 16, 16, 8
    h = 1.0 / nx
    rng = np.random.default_rng(4)
    shape = (nz, nx, ny)
    b = rng.standard_normal(shape).astype(np.float32)
    sdf = (rng.standard_normal(shape) * 0.1).astype(np.float32)
    p = rng.standard_normal(shape).astype(np.float32)
    net = wp.UNetWarmStart((nx, ny, nz), seed=3)
    params = net.params(0).astype(np.float64)
    # forward
    pred = torch.empty(shape, device="cuda")
    net.predict(pred, T(b), T(sdf), h)
    torch.cuda.synchronize()
    ref_pred, _ = oracle.unet_forward(params, b, sdf, h)
    assert rel(ref_pred, pred.cpu().numpy()) < 3e-2, rel(ref_pred, pred.cpu().numpy())
    # loss and gradients (lr = 0: no update)
    loss = net.train_step(T(b), T(sdf), T(p), h, 0.0)
    grads = net.params(1).astype(np.float64)
    # (1) against the oracle with the GPU's BF16 storage points emulated: per layer within 8e-2 (FP32
    # against FP64 accumulation still flips single BF16 roundings along the ~20 stored tensors, where
    # the plain FP64 oracle differs from the GPU by up to ~0.2 per layer)
    emu_loss, emu_grads = oracle.unet_loss_grad(params, b, sdf, p, h, bf16=True)
    assert abs(loss - emu_loss) < 1e-2 * emu_loss, (loss, emu_loss)
    for k, sl in enumerate(_groups(oracle)):
        if np.linalg.norm(emu_grads[sl]) > 0:
            assert rel(emu_grads[sl], grads[sl]) < 8e-2, (k, rel(emu_grads[sl], grads[sl]))
    # (2) against the exact FP64 gradient: the same descent direction
    ref_loss, ref_grads = oracle.unet_loss_grad(params, b, sdf, p, h)
    assert abs(loss - ref_loss) < 2e-2 * ref_loss, (loss, ref_loss)
    cos = float(np.dot(grads, ref_grads) / (np.linalg.norm(grads) * np.linalg.norm(ref_grads)))
    assert cos > 0.99, cos
    assert np.array_equal(net.params(0).astype(np.float64), params)  # lr = 0 left the weights alone


def test_unet_adam_step_changes_weights_and_roundtrips(wp):
    net = wp.UNetWarmStart((16, 16, 8), seed=1)
    v0 = net.params(0)
    b = torch.randn((8, 16, 16), device="cuda")
    sdf = torch.ones((8, 16, 16), device="cuda")
    loss0 = net.train_step(b, sdf, b * 0.01, 1 / 16, 1e-3)
    v1 = net.params(0)
    assert np.isfinite(loss0) and not np.array_equal(v0, v1)
    net.set_params(v0)
    assert np.array_equal(net.params(0), v0)
    with pytest.raises(wp.WPError):
        wp.UNetWarmStart((24, 16, 8))  # nx not a power of two


def test_device_velocity_generator(wp, oracle):
    dim = (32, 16, 24)
    s = wp.mac_shapes3d(*dim)
    u1 = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
    u2 = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
    wp.velocity3d_device(*u1, dim, seed=5)
    wp.velocity3d_device(*u2, dim, seed=5)
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(u1, u2))
    wp.velocity3d_device(*u2, dim, seed=6)
    assert not torch.equal(u1[0], u2[0])
    # walls closed; with phi switched off the field is a discrete curl, divergence-free in every cell
    # that does not touch a wall (the zeroed wall faces carry the curl's wall flux)
    assert float(u1[0][:, 0].abs().max()) == 0.0 and float(u1[2][-1].abs().max()) == 0.0
    wp.velocity3d_device(*u2, dim, seed=5, phi_rms=0.0)
    d = oracle.divergence3d(*[t.double().cpu().numpy() for t in u2],
                            *[np.ones(s[k]) for k in ("xv", "yv", "zv")], dim, (1 / 32, 1 / 16, 1 / 24))
    scale = max(float(t.abs().max()) for t in u2) * 32
    assert np.max(np.abs(d[1:-1, 1:-1, 1:-1])) < 1e-5 * scale
    assert np.max(np.abs(d)) > 1e-3 * scale  # the wall cells do see the closed faces
    f = torch.empty((24, 32, 16), device="cuda")
    wp.random_field3d(f, -2.0, 0.5, kmax=8, seed=1)
    assert abs(float(f.std()) - 0.5) < 0.15


def test_trained_warm_start_learns_and_fallback_bounds_its_cost(wp):
    """What the trained network does, stated as it is: training on the plain method's solves halves
    the loss; on held-out 32^3 problems the solve still meets its tolerance; the guess beats a zero
    start after one V-cycle; and the fallback (decided after that cycle) keeps the cost at most one
    cycle above the plain method.  The guess does not save cycles here or at 128^3 (the warm-start
    run summary in profiles/), so no test asserts that it does."""
    from waveletpotentials_b200 import trainer
    dim = (32, 32, 32)
    train = trainer.make_dataset(dim, 12, seed=1)
    held = trainer.make_dataset(dim, 4, seed=99)
    net = wp.UNetWarmStart(dim, seed=0)
    losses = trainer.train(net, train, steps=300, lr=3e-3, lr_end=3e-4)
    assert np.mean(losses[-30:]) < 0.5 * np.mean(losses[:5]), (losses[:5], losses[-30:])
    res = trainer.evaluate(net, held, tol=1e-6)
    plain = np.mean([r["plain_cycles"] for r in res])
    warm = np.mean([r["warm_cycles"] for r in res])
    print("warm start at 32^3:", res)
    # the tolerance is met either way; the fallback bounds the loss to the one discarded cycle
    assert all(r["warm_rel_residual"] <= 1e-6 for r in res)
    assert warm <= plain + 1.0, (plain, warm)
    # the trained guess beats a zero start after one V-cycle on average
    assert np.mean([r["warm_first_cycle"] for r in res]) < np.mean([r["plain_first_cycle"] for r in res])
