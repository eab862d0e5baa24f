"""Stage times of the reference CUDA build next to this build's on one GPU (test infrastructure).

The 256^3 benchmark input (four spheres, seed 0): the reference's V-cycle (piecewise-constant
prolongation, V(2,2), omega 2/3, CuMultigridFrac3D::Solve), its gradient update, and its wavelet
recovery (CuWaveletPotentialRecover3D::Solve) from ref_driver bench3d, FP64 (the reference default)
and FP32; beside them the same reference cycle in this build (wp_mgfrac3d_solve in FP32,
wp_mgfrac3d_solve_tol with WP_PROLONG_CONSTANT in FP64, autotuned), its wavelet recovery and its
fused gradient update.  Prints one JSON line.

    python oracle/refharness/compare_same_box.py [--n 256] [--cycles 4] [--reps 3]
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


def reference(driver, n, u, a, cycles, reps):
    with tempfile.TemporaryDirectory() as tin, tempfile.TemporaryDirectory() as tout:
        for k, v in zip(("xv", "yv", "zv", "ax", "ay", "az"), (*u, *a)):
            np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(tin, k + ".bin"))
        out = subprocess.run([driver, "bench3d", tin, tout, str(n), str(cycles), "2", "2", str(2.0 / 3.0), str(reps)],
                             check=True, timeout=3000, stdout=subprocess.PIPE, text=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def ours(n, u, a, cycles, reps):
    import torch
    from waveletpotentials_b200 import api
    nn = (n, n, n)
    h = 1.0 / n
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32, device="cuda")  # noqa: E731
    tu, ta = [T(x) for x in u], [T(x) for x in a]
    s = api.mac_shapes3d(*nn)
    b = torch.empty(s["p"], device="cuda")
    api.CuConvergence.GetB_3d_frac_vel(b, *tu, *ta, nn, h)
    mg = api.CuMultigridFrac3D(*ta, nn, h)
    mg.Autotune()
    p = torch.zeros(s["p"], device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    r = {}
    r["ms_per_cycle_fp32"] = timed(lambda: mg.Solve(p, None, b, cycles, 2, 2, 2.0 / 3.0)) / cycles
    r["ms_per_cycle_fp64"] = timed(lambda: mg.SolveTol(p, None, b, rel_tol=0.0, max_cycles=cycles, nu1=2, nu2=2,
                                                       weight=2.0 / 3.0, precision=api.PREC_FP64,
                                                       prolongation=api.PROLONG_CONSTANT,
                                                       raise_on_fail=False)) / cycles
    rec = api.CuWaveletPotentialRecover3D(nn, h)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    r["ms_recovery"] = timed(lambda: rec.Solve(*q, *tu))
    uu = [x.clone() for x in tu]
    r["ms_gradient_update"] = timed(lambda: api.CuGradient.SubtractGradient3D_Frac_P(*uu, p, *ta, nn, h))
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--cycles", type=int, default=4)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    import bench
    from oracle import oracle as O
    n = args.n
    centers, radii, u = bench.make_problem(n, 0)
    sdf = O.sdf_spheres3d((n, n, n), 1.0 / n, centers, radii)
    a = [x.astype(np.float32).astype(np.float64) for x in O.fractions3d(sdf, (n, n, n), 1.0 / n)]
    u = [np.asarray(x, np.float64) for x in u]
    res = {"n": n, "cycles": args.cycles, "input": "256^3 benchmark field, 4 spheres, seed 0"}
    for tag, drv in (("fp64", "ref_driver"), ("fp32", "ref_driver_f32")):
        path = os.path.join(ROOT, "oracle", "_ref", drv)
        if os.path.exists(path):
            rr = reference(path, n, u, a, args.cycles, args.reps)
            res[f"reference_{tag}"] = {"ms_per_cycle": rr["ms_divergence_and_solve"] / args.cycles,
                                       "ms_recovery": rr["ms_recovery"],
                                       "ms_gradient_update_maxdiv": rr["ms_gradient_update_maxdiv"],
                                       "ms_projection": rr["ms_mean"], "rel_residual": rr["rel_residual"]}
    res["ours"] = ours(n, u, a, args.cycles, args.reps)
    o = res["ours"]
    for tag in ("fp64", "fp32"):
        if f"reference_{tag}" in res:
            rf = res[f"reference_{tag}"]
            res[f"ratio_{tag}"] = {"cycle": rf["ms_per_cycle"] / o[f"ms_per_cycle_{tag}"],
                                   "recovery": rf["ms_recovery"] / o["ms_recovery"]}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
