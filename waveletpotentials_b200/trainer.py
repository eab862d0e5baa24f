"""Training data and training loop of the warm-start U-Net (config: 1-8 random spheres and boxes,
sizes U(0.05, 0.2), velocity u = curl(psi) + grad(phi) from the device generator).

A sample is one pressure solve of the plain method: b = -div(a u), the mixed-precision fractional
multigrid to the given tolerance, and the solid level set; the network learns b, sdf -> p.  Every
step runs on the GPU through the library (generator, solids, divergence, multigrid, the network's
forward/backward/Adam); this module only sequences the calls.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import api, fields


def make_sample(dim, seed: int, tol: float = 1e-6, kmax: int = 8):
    """One solved problem as device tensors {b, sdf, p, cycles, fractions}."""
    nx, ny, nz = dim
    h = 1.0 / nx
    s = api.mac_shapes3d(nx, ny, nz)
    centers, radii, lo, hi = fields.random_obstacles(seed, nmin=1, nmax=8, smin=0.05, smax=0.2)
    sls = api.CuSolidLevelSet3D(dim, h)
    sls.InitLsSpheres(centers, radii)
    if len(lo):
        sls.AddBoxes(lo, hi)
    a = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
    sls.GetFrac(*a)
    u = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
    api.velocity3d_device(*u, dim, seed=seed + 7919, kmax=kmax)
    b = torch.empty(s["p"], device="cuda")
    api.CuConvergence.GetB_3d_frac_vel(b, *u, *a, dim, h)
    mg = api.CuMultigridFrac3D(*a, dim, h)
    p = torch.zeros(s["p"], device="cuda")
    rep = mg.SolveTol(p, None, b, rel_tol=tol, max_cycles=60, precision=api.PREC_MIXED, raise_on_fail=False)
    return {"b": b, "sdf": sls.ls.clone(), "p": p, "cycles": rep["cycles"], "a": a, "h": h, "mg": mg, "u": u,
            "dim": tuple(dim)}


def make_dataset(dim, count: int, seed: int = 0, tol: float = 1e-6):
    return [make_sample(dim, seed + 1000 * i, tol) for i in range(count)]


def train(net: api.UNetWarmStart, samples, steps: int, lr: float = 2e-3, lr_end: float = 2e-4, log_every: int = 0):
    """Adam steps over the samples in a seeded random order, cosine-decayed learning rate."""
    rng = np.random.default_rng(0)
    losses = []
    t0 = time.perf_counter()
    for k in range(steps):
        s = samples[int(rng.integers(len(samples)))]
        rate = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * k / max(steps - 1, 1)))
        losses.append(net.train_step(s["b"], s["sdf"], s["p"], s["h"], rate))
        if log_every and (k % log_every == 0 or k == steps - 1):
            print(f"step {k} loss {losses[-1]:.4g} lr {rate:.3g} ({time.perf_counter() - t0:.1f} s)", flush=True)
    return losses


def evaluate(net: api.UNetWarmStart, samples, tol: float = 1e-6):
    """V-cycles to `tol` from a zero start and from the network's guess (with the fallback rule of
    Projector3D: the guess is used only if its residual is below the zero start's)."""
    out = []
    opts = dict(rel_tol=tol, max_cycles=60, precision=api.PREC_MIXED)
    for s in samples:
        mg = s["mg"]
        dst = torch.zeros_like(s["b"])
        plain = mg.SolveTol(dst, None, s["b"], raise_on_fail=False, **opts)
        guess = torch.empty_like(s["b"])
        net.predict(guess, s["b"], s["sdf"], s["h"])
        r0 = mg.GetResdualError(guess, s["b"])
        warm = api.warm_started_solve(mg, dst, s["b"], s["sdf"], s["h"], net, opts)
        out.append({"plain_cycles": plain["cycles"], "warm_cycles": warm["cycles"], "initial_rel_residual": r0,
                    "plain_first_cycle": plain["history"][0] if plain["history"] else None,
                    "warm_first_cycle": warm["warm_start"]["first_cycle_rel_residual"],
                    "used": warm["warm_start"]["used"], "warm_rel_residual": warm["rel_residual"]})
    return out
