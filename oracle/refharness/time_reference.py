"""Time the reference CUDA build on one projection (test infrastructure, GPU host only).

One projection = b = -div(a u) -> CuMultigridFrac3D::Solve -> u <- a (u - grad p) -> max|div| ->
CuWaveletPotentialRecover3D::Solve, the composition of TestLocalProjection.cpp:666-767.  The cycle
count is the first V-cycle count whose relative residual reaches the tolerance, found with the
reference's own per-cycle residual (CuMultigridFrac3D::GetResdualError).

    python oracle/refharness/time_reference.py --n 128 --tol 1e-6 [--driver oracle/_ref/ref_driver]

With --index-fluid F it times instead four V(2,2) cycles (omega 0.8) of CuMultigridFrac3D::Solve_index
and of CuMultigridFrac3D::Solve on the mostly-solid domain the bench uses for the index-sparse cycle
(waveletpotentials_b200.fields.porous_domain with fluid fraction F, right-hand side random on the
fluid cells), best of --reps calls of each:

    python oracle/refharness/time_reference.py --n 256 --index-fluid 0.15

The reference's coarsest kernel (cuWjFrac3D_kernel_n) holds at most 512 cells, so the index run
is refused unless every level lists a cell (the cycle then ends on the 2^3 level).

Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from waveletpotentials_b200 import fields  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--nu", type=int, default=2)
    ap.add_argument("--omega", type=float, default=2.0 / 3.0)
    ap.add_argument("--spheres", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-cycles", type=int, default=60)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--driver", default=os.path.join(ROOT, "oracle", "_ref", "ref_driver"))
    ap.add_argument("--index-fluid", type=float, default=0.0)
    a = ap.parse_args()
    n = a.n
    nn = (n, n, n)
    if a.index_fluid > 0:
        return time_index(a, nn)
    if a.spheres == 1:
        centers, radii = np.array([[0.5, 0.5, 0.5]]), np.array([0.2])
    else:
        centers, radii = fields.random_spheres(a.spheres, 0.05, 0.15, a.seed + 1000)
    sdf = O.sdf_spheres3d(nn, 1.0 / n, centers, radii)
    ax, ay, az = O.fractions3d(sdf, nn, 1.0 / n)
    xv, yv, zv = fields.velocity3d(nn, a.seed)
    with tempfile.TemporaryDirectory() as tin, tempfile.TemporaryDirectory() as tout:
        for k, v in dict(xv=xv, yv=yv, zv=zv, ax=ax, ay=ay, az=az).items():
            np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(tin, k + ".bin"))
        f = O.divergence3d(xv, yv, zv, ax, ay, az, nn, (1.0 / n,) * 3)
        f.tofile(os.path.join(tin, "f.bin"))
        params = (n, n, n, 1.0 / n, a.max_cycles, a.nu, a.nu, a.omega)
        subprocess.run([a.driver, "mg3d", tin, tout] + [str(x) for x in params], check=True, timeout=3000)
        hist = np.fromfile(os.path.join(tout, "hist.bin"), dtype=np.float64)
        hit = np.nonzero(hist <= a.tol)[0]
        ncycles = int(hit[0]) + 1 if hit.size else a.max_cycles
        out = subprocess.run([a.driver, "bench3d", tin, tout] + [str(x) for x in
                                                                  (n, ncycles, a.nu, a.nu, a.omega, a.reps)],
                             check=True, timeout=3000, stdout=subprocess.PIPE, text=True).stdout
    res = json.loads(out.strip().splitlines()[-1])
    res.update({"tol": a.tol, "tol_reached": bool(hit.size), "history": [float(h) for h in hist[:ncycles]],
                "driver": os.path.basename(a.driver), "spheres": a.spheres})
    print(json.dumps(res))


def time_index(a, nn):
    n = nn[0]
    fl, (ax, ay, az), frng = fields.porous_domain(nn, a.index_fluid, a.seed)
    f = frng.standard_normal(fl.shape) * fl
    _, _, counts = O.mgfrac3d_solve_index(f, ax, ay, az, nn, (1.0 / n,) * 3, 0, 2, 2, 0.8)
    if not all(c > 0 for c in counts):
        sys.exit(f"a level lists no cell ({list(counts)}): the reference's coarsest kernel would take a level "
                 "of more than 512 cells")
    with tempfile.TemporaryDirectory() as tin, tempfile.TemporaryDirectory() as tout:
        for k, v in dict(f=f, ax=ax, ay=ay, az=az).items():
            np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(tin, k + ".bin"))
        params = (n, n, n, 1.0 / n, 4, 2, 2, 0.8, a.reps)
        subprocess.run([a.driver, "mg3d_index", tin, tout] + [str(x) for x in params], check=True, timeout=3000,
                       stdout=subprocess.DEVNULL)
        t = np.fromfile(os.path.join(tout, "timing.bin"), dtype=np.float64)
    print(json.dumps({"workload": f"{n}^3 cells, {fl.mean():.3f} fluid, 4 V(2,2) cycles, omega 0.8",
                      "listed_cells": [int(c) for c in counts], "index_ms_per_cycle": float(t[0]) / 4,
                      "dense_ms_per_cycle": float(t[1]) / 4, "driver": os.path.basename(a.driver)}))


if __name__ == "__main__":
    main()
