"""Seeded synthetic inputs: spectral Gaussian random fields on the MAC grid and random solids.

These are the benchmark inputs (no dataset exists for this method).  A velocity field is built as
``u = curl_h(psi) + grad_h(phi)`` with the discrete MAC curl of an edge potential (the operator of
the reference's host check, StreamInitial.cpp:87-175) and the face gradient of a cell-centred
scalar, so its divergence-free part is exactly representable.  Wall-normal faces are zero
(zero-normal-flux walls, as the reference's input generator leaves them: TestLocalProjection.cpp:185-221).

Arrays follow the reference layout: a 3D array with extents (DX, DY, DZ) has numpy shape
(DZ, DX, DY), y fastest; 2D arrays are (DX, DY).
"""
from __future__ import annotations

import numpy as np


def spectral_field(shape, slope: float, rms: float, rng: np.random.Generator) -> np.ndarray:
    """Gaussian random field with isotropic power spectrum P(k) ~ k^slope, scaled to the given RMS."""
    white = rng.standard_normal(shape)
    spec = np.fft.rfftn(white)
    ks = [np.fft.fftfreq(s) for s in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    k2 = np.zeros(spec.shape)
    for ax, k in enumerate(ks):
        sh = [1] * len(shape)
        sh[ax] = k.size
        k2 = k2 + (k.reshape(sh) * shape[ax]) ** 2
    kk = np.sqrt(k2)
    kk.flat[0] = 1.0
    amp = kk ** (slope / 2.0)
    amp.flat[0] = 0.0
    field = np.fft.irfftn(spec * amp, s=shape, axes=tuple(range(len(shape))))
    std = float(field.std())
    return field * (rms / std if std > 0 else 0.0)


def curl3d(qx, qy, qz, n, d):
    """Discrete curl of an edge potential onto MAC faces (StreamInitial.cpp:87-143)."""
    nx, ny, nz = n
    dx, dy, dz = d
    xv = (qz[:, :, 1:] - qz[:, :, :-1]) / dy - (qy[1:, :, :] - qy[:-1, :, :]) / dz
    yv = (qx[1:, :, :] - qx[:-1, :, :]) / dz - (qz[:, 1:, :] - qz[:, :-1, :]) / dx
    zv = (qy[:, 1:, :] - qy[:, :-1, :]) / dx - (qx[:, :, 1:] - qx[:, :, :-1]) / dy
    return xv, yv, zv


def curl2d(qz, n, d):
    """2D stream-function curl (StreamInitial.cpp:145-175)."""
    dx, dy = d
    xv = (qz[:, 1:] - qz[:, :-1]) / dy
    yv = -(qz[1:, :] - qz[:-1, :]) / dx
    return xv, yv


def velocity3d(n, seed: int, psi_slope=-11.0 / 3.0, psi_rms=1.0, phi_slope=-2.0, phi_rms=1.0, dtype=np.float64):
    """u = curl(psi) + grad(phi) on an nx*ny*nz MAC grid over the unit domain (dx = 1/n)."""
    nx, ny, nz = n
    d = (1.0 / nx, 1.0 / ny, 1.0 / nz)
    rng = np.random.default_rng(seed)
    big = (nz + 1, nx + 1, ny + 1)
    qx = spectral_field(big, psi_slope, psi_rms, rng)[:, :nx, :]
    qy = spectral_field(big, psi_slope, psi_rms, rng)[:, :, :ny]
    qz = spectral_field(big, psi_slope, psi_rms, rng)[:nz, :, :]
    xv, yv, zv = curl3d(qx, qy, qz, n, d)
    phi = spectral_field((nz, nx, ny), phi_slope, phi_rms, rng)
    xv[:, 1:-1, :] += (phi[:, 1:, :] - phi[:, :-1, :]) / d[0]
    yv[:, :, 1:-1] += (phi[:, :, 1:] - phi[:, :, :-1]) / d[1]
    zv[1:-1, :, :] += (phi[1:, :, :] - phi[:-1, :, :]) / d[2]
    xv[:, 0, :] = xv[:, -1, :] = 0.0
    yv[:, :, 0] = yv[:, :, -1] = 0.0
    zv[0] = zv[-1] = 0.0
    return (np.ascontiguousarray(xv, dtype=dtype), np.ascontiguousarray(yv, dtype=dtype),
            np.ascontiguousarray(zv, dtype=dtype))


def velocity2d(n, seed: int, psi_slope=-3.0, psi_rms=1.0, phi_slope=-2.0, phi_rms=0.5, dtype=np.float64):
    nx, ny = n
    d = (1.0 / nx, 1.0 / ny)
    rng = np.random.default_rng(seed)
    psi = spectral_field((nx + 1, ny + 1), psi_slope, psi_rms, rng)
    xv, yv = curl2d(psi, n, d)
    phi = spectral_field((nx, ny), phi_slope, phi_rms, rng)
    xv[1:-1, :] += (phi[1:, :] - phi[:-1, :]) / d[0]
    yv[:, 1:-1] += (phi[:, 1:] - phi[:, :-1]) / d[1]
    xv[0] = xv[-1] = 0.0
    yv[:, 0] = yv[:, -1] = 0.0
    return np.ascontiguousarray(xv, dtype=dtype), np.ascontiguousarray(yv, dtype=dtype)


def random_spheres(count: int, rmin: float, rmax: float, seed: int):
    """Sphere centres/radii inside the unit cube (each sphere fully inside the domain)."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(rmin, rmax, count)
    centers = np.stack([rng.uniform(r + 0.02, 1.0 - r - 0.02, 3) for r in radii]) if count else np.zeros((0, 3))
    return centers, radii


def random_obstacles(seed: int, nmin=1, nmax=8, smin=0.05, smax=0.2):
    """Mixed spheres and axis-aligned boxes (sizes uniform in [smin, smax])."""
    rng = np.random.default_rng(seed)
    count = int(rng.integers(nmin, nmax + 1))
    centers, radii, lo, hi = [], [], [], []
    for _ in range(count):
        size = rng.uniform(smin, smax)
        c = rng.uniform(size + 0.05, 1.0 - size - 0.05, 3)
        if rng.random() < 0.5:
            centers.append(c)
            radii.append(size)
        else:
            half = rng.uniform(0.5, 1.0, 3) * size
            lo.append(c - half)
            hi.append(c + half)
    return (np.array(centers).reshape(-1, 3), np.array(radii), np.array(lo).reshape(-1, 3),
            np.array(hi).reshape(-1, 3))


def sdf_spheres3d(n, centers, radii):
    """Signed distance to a union of spheres at cell centres, positive in fluid
    (cuInitLsSphere, cuSolidLevelSet3D.cu:11-27)."""
    nx, ny, nz = n
    h = 1.0 / nx
    z, x, y = np.meshgrid((np.arange(nz) + 0.5) * h, (np.arange(nx) + 0.5) * h, (np.arange(ny) + 0.5) * h,
                          indexing="ij")
    out = np.full((nz, nx, ny), 1e30)
    for c, r in zip(np.reshape(centers, (-1, 3)), np.reshape(radii, (-1,))):
        out = np.minimum(out, np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r)
    return out


def porous_fractions(fluid, rng, tiny=0, cut=True):
    """Face fractions of a cell mask (numpy (nz, nx, ny), True = fluid): 1 between two fluid cells, a
    random value in [0.2, 0.9] between a fluid and a solid cell (0 with cut=False), 0 between two
    solid cells; a wall face takes its cell's value.  `tiny` faces of solid-solid pairs get 1e-13
    (below the 1e-12 threshold of the index-sparse cycle's cell selection).  Returns (ax, ay, az)."""
    m = fluid.astype(np.float64)
    out = []
    for axis in (1, 2, 0):  # ax (x faces), ay (y faces), az (z faces)
        pad = np.concatenate([np.take(m, [0], axis=axis), m, np.take(m, [-1], axis=axis)], axis=axis)
        lo = np.take(pad, range(0, pad.shape[axis] - 1), axis=axis)
        hi = np.take(pad, range(1, pad.shape[axis]), axis=axis)
        part = rng.uniform(0.2, 0.9, lo.shape) if cut else np.zeros(lo.shape)
        a = np.where((lo > 0) & (hi > 0), 1.0, np.where((lo > 0) | (hi > 0), part, 0.0))
        if tiny:
            zero = np.argwhere(a == 0.0)
            pick = zero[rng.choice(len(zero), size=min(tiny, len(zero)), replace=False)]
            a[tuple(pick.T)] = 1e-13
        out.append(a)
    return out


def porous_domain(n, fluid_fraction: float, seed: int, rmin=0.04, rmax=0.1):
    """A mostly-solid domain for the index-sparse multigrid: balls of fluid (radii uniform in
    [rmin, rmax] of the extent) dropped until `fluid_fraction` of the cells are fluid, with cut faces
    of random area where fluid meets solid.  Returns (fluid mask, (ax, ay, az), rng)."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    z, x, y = np.meshgrid(np.arange(nz) + 0.5, np.arange(nx) + 0.5, np.arange(ny) + 0.5, indexing="ij",
                          sparse=True)
    fluid = np.zeros((nz, nx, ny), dtype=bool)
    ext = np.array([nx, ny, nz], dtype=np.float64)
    while fluid.mean() < fluid_fraction:
        c = rng.uniform(0, 1, 3) * ext
        r = rng.uniform(rmin, rmax) * min(n)
        fluid |= (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 < r * r
    return fluid, porous_fractions(fluid, rng), rng
