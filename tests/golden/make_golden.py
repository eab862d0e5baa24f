"""Generate the golden fixtures in this directory from the reference's own CUDA build.

Run on a GPU host after ``make -C oracle/refharness`` has built ``oracle/_ref/ref_driver`` from the
unmodified reference sources (FP64, the reference default):

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --only index   # the index-sparse multigrid cases only
    python tests/golden/make_golden.py --only cut     # the coefficient truncation cases only
    python tests/golden/make_golden.py --only frac    # the sub-sampled face fraction cases only
    python tests/golden/make_golden.py --only sweep   # the fast sweeping cases only
    python tests/golden/make_golden.py --only cdf35   # the CDF3.5 transforms only
    python tests/golden/make_golden.py --only dst     # CuDst3D::Solve only
    python tests/golden/make_golden.py --only psweep  # CuParallelSweep3D Solve / Project only
    python tests/golden/make_golden.py --only domd    # projection and recovery with Dirichlet walls
    python tests/golden/make_golden.py --only families  # CDF2.6 / CDF2.8 / CDF4.4 transforms
    python tests/golden/make_golden.py --only short   # CDF2.0 / CDF1.1 / CDF1.7 transforms
    python tests/golden/make_golden.py --only domd2d  # 2D projection and recovery with Dirichlet walls
    python tests/golden/make_golden.py --only narrow  # CuFastSweeping::ParticlesToLsNarrow
    python tests/golden/make_golden.py --only psweep_d  # CuParallelSweep3D with bc 'd'
    python tests/golden/make_golden.py --only psweep_mid  # CuParallelSweep3D::SolveFromMid
    ... [--out DIR]                                   # write the .npz files to DIR instead of here

Every case draws seeded inputs with numpy, runs the reference entry point through ref_driver
(CuWHHDForward::Solve1D, CuGetInnerProduct::GenerateIp, CuDivLocalProject3D::ProjectLocal_q_ccc,
CuDivLocalProject::ProjectSingle, CuWaveletPotentialRecover3D/2D::Solve, CuMultigridFrac3D/2D::Solve,
CuMultigridFrac3D::Solve_index, CuWaveletPotentialRecover3D::CutCoefficients, CuSolidLevelSet3D::GetFrac (static, sub-sampled), CuFastSweeping (incl. ParticlesToLs),
CuConvergence::GetB_3d_frac_vel, CuGradient::Gradient3D_Frac_P,
CuSolidLevelSet3D) and stores inputs
and reference outputs as ``<case>.npz``.  The CPU tests pin the FP64 oracle against these files;
the GPU tests compare the CUDA kernels with the oracle on the same inputs.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from waveletpotentials_b200.fields import porous_fractions  # noqa: E402
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
DRIVER32 = os.path.join(ROOT, "oracle", "_ref", "ref_driver_f32")
CDF3_5, CDF2_6, CDF4_4, CDF4_6, CDF2_8, CDF3_7 = 2, 5, 6, 7, 10, 11
CDF2_0, CDF1_1, CDF1_7 = 16, 17, 18


def run(op, inputs: dict, params, outputs: dict, driver=None):
    """inputs: name -> array; outputs: name -> shape. Returns dict of output arrays.  driver: the
    FP64 build (default) or DRIVER32."""
    with tempfile.TemporaryDirectory() as tin, tempfile.TemporaryDirectory() as tout:
        for k, v in inputs.items():
            np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(tin, k + ".bin"))
        cmd = [driver or DRIVER, op, tin, tout] + [str(p) for p in params]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=600, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
            raise subprocess.CalledProcessError(r.returncode, cmd)
        return {k: np.fromfile(os.path.join(tout, k + ".bin"), dtype=np.float64).reshape(s)
                for k, s in outputs.items()}


OUT_DIR = HERE


def save(name, **arrays):
    np.savez_compressed(os.path.join(OUT_DIR, name + ".npz"), **arrays)
    print("wrote", name, {k: np.shape(v) for k, v in arrays.items()})


def shapes3(n):
    nx, ny, nz = n
    return {"xv": (nz, nx + 1, ny), "yv": (nz, nx, ny + 1), "zv": (nz + 1, nx, ny),
            "qx": (nz + 1, nx, ny + 1), "qy": (nz + 1, nx + 1, ny), "qz": (nz, nx + 1, ny + 1), "p": (nz, nx, ny)}


def index_cases(rng):
    """CuMultigridFrac3D::Solve_index on mostly-solid domains: tubes and a sphere in a non-cubic box,
    a fluid island whose coarse level lists no cell (the cycle stops at the finest level), and the
    inside of a sphere (the reference's own fractions, inverted)."""
    n = (24, 20, 18)
    nx, ny, nz = n
    z, x, y = np.meshgrid(np.arange(nz) + 0.5, np.arange(nx) + 0.5, np.arange(ny) + 0.5, indexing="ij")
    fluid = ((x - 7) ** 2 + (y - 9) ** 2 < 9) | ((z - 5) ** 2 + (y - 13) ** 2 < 6) | \
            ((x - 16) ** 2 + (y - 6) ** 2 + (z - 11) ** 2 < 20)
    cases = [("mg3d_index_pores", n, fluid, 40, True, 4, (2, 3), 0.8)]
    # the cycle stops at the finest level; the reference's coarsest kernel (cuWjFrac3D_kernel_n) holds
    # at most 512 cells (one CTA of shared memory), so the island case stays at 8^3
    isl = np.zeros((8, 8, 8), dtype=bool)
    isl[2:4, 4:6, 2:4] = True
    cases.append(("mg3d_index_island", (8, 8, 8), isl, 0, False, 3, (2, 2), 0.8))
    for tag, nn, fl, tiny, cut, cyc, nu, w in cases:
        ax, ay, az = porous_fractions(fl, rng, tiny, cut)
        f = rng.standard_normal(fl.shape)
        out = run("mg3d_index", {"f": f, "ax": ax, "ay": ay, "az": az}, [*nn, 1.0 / nn[0], cyc, nu[0], nu[1], w],
                  {"p": fl.shape, "hist": (cyc,)})
        save(tag, n=np.array(nn), h=1.0 / nn[0], f=f, ax=ax, ay=ay, az=az, ncycles=cyc, nu=np.array(nu), omega=w,
             **out)
    n3 = 32
    s = shapes3((n3, n3, n3))
    fr = run("frac3d", {}, [n3, 1.0 / n3, 0.5, 0.5, 0.45, 0.4], {k: s[k2] for k, k2 in
                                                                (("ax", "xv"), ("ay", "yv"), ("az", "zv"))})
    ax, ay, az = (1.0 - fr[k] for k in ("ax", "ay", "az"))
    f = rng.standard_normal(s["p"])
    out = run("mg3d_index", {"f": f, "ax": ax, "ay": ay, "az": az}, [n3, n3, n3, 1.0 / n3, 3, 2, 2, 2.0 / 3.0],
              {"p": s["p"], "hist": (3,)})
    save("mg3d_index_sphere32", n=np.array([n3] * 3), h=1.0 / n3, f=f, ax=ax, ay=ay, az=az, ncycles=3,
         nu=np.array([2, 2]), omega=2.0 / 3.0, **out)


def cut_cases(rng):
    """CuWaveletPotentialRecover3D::CutCoefficients on random potentials whose samples on the walls
    of the CDF4.6 (Dirichlet-type) axes are zero, at every level from 0 (the identity) to the
    smallest log2 extent, on a cube and a box."""
    out = {}
    for n in ((16, 16, 16), (16, 8, 32)):
        s = shapes3(n)
        q = {k: rng.standard_normal(s[k]) for k in ("qx", "qy", "qz")}
        q["qx"][:, :, [0, -1]] = 0
        q["qx"][[0, -1]] = 0
        q["qy"][:, [0, -1], :] = 0
        q["qy"][[0, -1]] = 0
        q["qz"][:, [0, -1], :] = 0
        q["qz"][:, :, [0, -1]] = 0
        tag = "x".join(str(v) for v in n)
        out[f"n_{tag}"] = np.array(n)
        for k in ("qx", "qy", "qz"):
            out[f"{k}_{tag}"] = q[k]
        for level in range(int(np.log2(min(n))) + 1):
            res = run("cut3d", q, [*n, 1.0 / n[0], level], {k: s[k] for k in ("qx", "qy", "qz")})
            for k in ("qx", "qy", "qz"):
                out[f"{k}_{tag}_cut{level}"] = res[k]
    save("cut3d", **out)


def frac_cases(rng):
    """The static CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx): sub-sampled face fractions of
    two level sets given as FP32 values -- two overlapping spheres in a box, and a wavy surface."""
    out = {}
    for tag, n in (("spheres", (24, 20, 16)), ("wavy", (16, 16, 16))):
        nx, ny, nz = n
        h = 1.0 / nx
        z, x, y = np.meshgrid((np.arange(nz) + 0.5) * h, (np.arange(nx) + 0.5) * h, (np.arange(ny) + 0.5) * h,
                              indexing="ij")
        if tag == "spheres":
            ls = np.minimum(np.sqrt((x - 0.45) ** 2 + (y - 0.4) ** 2 + (z - 0.3) ** 2) - 0.22,
                            np.sqrt((x - 0.7) ** 2 + (y - 0.55) ** 2 + (z - 0.35) ** 2) - 0.15)
        else:
            ls = z - 0.5 - 0.12 * np.sin(2 * np.pi * x * 1.5) * np.cos(2 * np.pi * y) + 0.01 * rng.standard_normal(x.shape)
        ls = ls.astype(np.float32).astype(np.float64)
        s = shapes3(n)
        res = run("frac3d_sub", {"ls": ls}, [nx, ny, nz, h], {"ax": s["xv"], "ay": s["yv"], "az": s["zv"]})
        out[f"n_{tag}"] = np.array(n)
        out[f"ls_{tag}"] = ls
        for k in ("ax", "ay", "az"):
            out[f"{k}_{tag}"] = res[k]
    save("frac3d_sub", **out)


def sweep_cases(rng):
    """CuFastSweeping::ReinitLevelSet on a squeezed, wavy sphere level set and CuFastSweeping::Solve
    from fixed negative sources with every other cell at +5, both run past convergence (the
    reference updates in place from concurrent threads, so only its fixed point is reproducible)."""
    n = (24, 20, 16)
    nx, ny, nz = n
    h = 1.0 / nx
    z, x, y = np.meshgrid((np.arange(nz) + 0.5) * h, (np.arange(nx) + 0.5) * h, (np.arange(ny) + 0.5) * h,
                          indexing="ij")
    sdf = np.sqrt((x - 0.5) ** 2 + (y - 0.45) ** 2 + (z - 0.4) ** 2) - 0.25
    ls1 = (0.6 * sdf + 0.01 * np.sin(9 * x) * np.cos(7 * y)).astype(np.float32).astype(np.float64)
    ls2 = np.where(sdf < 0, sdf, 5.0).astype(np.float32).astype(np.float64)
    r1 = run("fsweep", {"ls": ls1}, [nx, ny, nz, h, 80, 1], {"ls": ls1.shape})["ls"]
    r2 = run("fsweep", {"ls": ls2}, [nx, ny, nz, h, 80, 0], {"ls": ls2.shape})["ls"]
    # CuFastSweeping::ParticlesToLs: a blob of particles well inside the box (the reference does not
    # bound-check the cells around a particle)
    pts = (np.array([0.5, 0.45, 0.5]) + 0.12 * rng.standard_normal((60, 3))).clip(0.2, 0.8)
    pts = pts * np.array([nx, ny, nz]) * h
    pts = pts.astype(np.float32).astype(np.float64)
    r3 = run("p2ls", {"xyz": pts}, [nx, ny, nz, h, 0.6 * h, 1.0, 80, len(pts)], {"ls": ls1.shape})["ls"]
    save("fsweep", n=np.array(n), h=h, iters=80, ls_reinit=ls1, out_reinit=r1, ls_solve=ls2, out_solve=r2,
         particles=pts, radius=0.6 * h, max_dis=1.0, out_particles=r3)


def narrow_cases(rng):
    """CuFastSweeping::ParticlesToLsNarrow (cuFastSweeping.cu:352-385): the caller's level set is the
    start (no fill), lowered by the particles' rough distances, swept, negated and swept again; from a
    constant band value and from a wavy sphere level set, past convergence (the reference sweeps in
    place from concurrent threads, so only its fixed point is reproducible), with the particles well
    inside the box (the reference does not bound-check the cells around a particle)."""
    n = (24, 20, 16)
    nx, ny, nz = n
    h = 1.0 / nx
    z, x, y = np.meshgrid((np.arange(nz) + 0.5) * h, (np.arange(nx) + 0.5) * h, (np.arange(ny) + 0.5) * h,
                          indexing="ij")
    sdf = np.sqrt((x - 0.45) ** 2 + (y - 0.5) ** 2 + (z - 0.35) ** 2) - 0.2
    starts = {"band": np.full(sdf.shape, 4 * h), "wavy": 0.8 * sdf + 0.01 * np.sin(8 * x) * np.cos(6 * y)}
    out = {"n": np.array(n), "h": h, "iters": 80, "radius": 0.6 * h, "max_dis": 1.0}
    for tag, ls0 in starts.items():
        pts = (np.array([0.55, 0.5, 0.5]) + 0.1 * rng.standard_normal((50, 3))).clip(0.2, 0.8)
        pts = (pts * np.array([nx, ny, nz]) * h).astype(np.float32).astype(np.float64)
        ls0 = ls0.astype(np.float32).astype(np.float64)
        r = run("p2ls_narrow", {"xyz": pts, "ls": ls0}, [nx, ny, nz, h, 0.6 * h, 1.0, 80, len(pts)],
                {"ls": ls0.shape})["ls"]
        out.update({f"{tag}_particles": pts, f"{tag}_ls": ls0, f"{tag}_out": r})
    save("p2ls_narrow", **out)


def cdf35_cases(rng):
    """CuWHHDForward::Solve1D with CDF3.5 (another wavelet family of the same lifting structure):
    every axis, both boundary types, both directions, and a 256-point line."""
    dwt = {}
    for bc in "nd":
        for fwd in (1, 0):
            for axis, (L, other) in {"y": (4, (3, 2)), "x": (5, (4, 3)), "z": (3, (5, 2))}.items():
                n = 1 << L
                DX, DY, DZ = {"y": (other[0], n, other[1]), "x": (n, other[0], other[1]),
                              "z": (other[0], other[1], n)}[axis]
                a = rng.standard_normal((DZ, DX, DY))
                out = run("dwt1d", {"a": a}, [DX, DY, DZ, L, axis, bc, CDF3_5, fwd], {"c": (DZ, DX, DY)})
                key = f"w{CDF3_5}_{bc}_{'f' if fwd else 'i'}_{axis}"
                dwt[key + "_in"] = a
                dwt[key + "_out"] = out["c"]
                dwt[key + "_meta"] = np.array([DX, DY, DZ, L, ord(axis), ord(bc), CDF3_5, fwd])
        for fwd in (1, 0):
            a = rng.standard_normal((1, 2, 256))
            out = run("dwt1d", {"a": a}, [2, 256, 1, 8, "y", bc, CDF3_5, fwd], {"c": (1, 2, 256)})
            key = f"w{CDF3_5}_{bc}_{'f' if fwd else 'i'}_long"
            dwt[key + "_in"] = a
            dwt[key + "_out"] = out["c"]
            dwt[key + "_meta"] = np.array([2, 256, 1, 8, ord("y"), ord(bc), CDF3_5, fwd])
    save("dwt1d_cdf35", **dwt)


def families_cases(rng):
    """CuWHHDForward::Solve1D with the other whole-sample families the reference registers
    (cuWHHDForward.cu:788-870, 914-956): CDF2.6, CDF2.8 and CDF4.4 on lines of 2^L + 1 samples,
    every axis, the boundary types 'n', 'd' and 'z' (CDF2.x have a rule of their own for 'z', CDF4.4
    treats it as 'n'), both directions, and a 257-point line."""
    dwt = {}
    for wav in (CDF2_6, CDF2_8, CDF4_4):
        for bc in "ndz":
            for fwd in (1, 0):
                for axis, (L, other) in {"y": (4, (3, 2)), "x": (5, (4, 3)), "z": (3, (5, 2))}.items():
                    n = (1 << L) + 1
                    DX, DY, DZ = {"y": (other[0], n, other[1]), "x": (n, other[0], other[1]),
                                  "z": (other[0], other[1], n)}[axis]
                    a = rng.standard_normal((DZ, DX, DY))
                    out = run("dwt1d", {"a": a}, [DX, DY, DZ, L, axis, bc, wav, fwd], {"c": (DZ, DX, DY)})
                    key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_{axis}"
                    dwt[key + "_in"] = a
                    dwt[key + "_out"] = out["c"]
                    dwt[key + "_meta"] = np.array([DX, DY, DZ, L, ord(axis), ord(bc), wav, fwd])
                a = rng.standard_normal((1, 2, 257))
                out = run("dwt1d", {"a": a}, [2, 257, 1, 8, "y", bc, wav, fwd], {"c": (1, 2, 257)})
                key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_long"
                dwt[key + "_in"] = a
                dwt[key + "_out"] = out["c"]
                dwt[key + "_meta"] = np.array([2, 257, 1, 8, ord("y"), ord(bc), wav, fwd])
    save("dwt1d_families", **dwt)


def short_cases(rng):
    """CuWHHDForward::Solve1D with the short families the reference registers (cuWHHDForward.cu:
    998-1080): CDF2.0 (the CDF2.x predict alone, with CDF2.6's boundary rules, on lines of 2^L + 1)
    and CDF1.1 / CDF1.7 (a Haar predict and a 1- or 7-tap update, with CDF3.5's boundary rules, on
    lines of 2^L); every axis, the boundary types 'n' and 'd' (the only ones registered for these
    three), both directions, and a 256/257-point line."""
    dwt = {}
    for wav, ext in ((CDF2_0, 1), (CDF1_1, 0), (CDF1_7, 0)):
        for bc in "nd":
            for fwd in (1, 0):
                for axis, (L, other) in {"y": (4, (3, 2)), "x": (5, (4, 3)), "z": (3, (5, 2))}.items():
                    n = (1 << L) + ext
                    DX, DY, DZ = {"y": (other[0], n, other[1]), "x": (n, other[0], other[1]),
                                  "z": (other[0], other[1], n)}[axis]
                    a = rng.standard_normal((DZ, DX, DY))
                    out = run("dwt1d", {"a": a}, [DX, DY, DZ, L, axis, bc, wav, fwd], {"c": (DZ, DX, DY)})
                    key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_{axis}"
                    dwt[key + "_in"] = a
                    dwt[key + "_out"] = out["c"]
                    dwt[key + "_meta"] = np.array([DX, DY, DZ, L, ord(axis), ord(bc), wav, fwd])
                n = 256 + ext
                a = rng.standard_normal((1, 2, n))
                out = run("dwt1d", {"a": a}, [2, n, 1, 8, "y", bc, wav, fwd], {"c": (1, 2, n)})
                key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_long"
                dwt[key + "_in"] = a
                dwt[key + "_out"] = out["c"]
                dwt[key + "_meta"] = np.array([2, n, 1, 8, ord("y"), ord(bc), wav, fwd])
    save("dwt1d_short", **dwt)


def dst_cases(rng):
    """CuDst3D::Solve (the Dirichlet Poisson solve by DST-I along each axis, cuDst3D.cu:265-341) on
    grids of equal extents (its constructor's buffer sizing is only safe there, cuDst3D.cu:209-211):
    an even and an odd extent, unequal spacings."""
    out = {}
    for tag, n, d in (("15", 15, (1 / 16, 1 / 16, 1 / 16)), ("8", 8, (0.1, 0.07, 0.13))):
        f = rng.standard_normal((n, n, n))
        p = run("dst3d", {"f": f}, [n, n, n, *d], {"p": (n, n, n)})["p"]
        out[f"f_{tag}"], out[f"p_{tag}"], out[f"d_{tag}"] = f, p, np.array(d)
    save("dst3d", **out)


def psweep_cases(rng):
    """CuParallelSweep3D with bc 'n' (the reference's comparison baseline): Solve then Project on a
    divergence-free field with no flux through the walls, as TestLocalProjection.cpp:719-721 calls
    them, at 8^3 and 16^3 (a first 32^3 run in a fresh process left through the reference's CUDA
    error exit and was not repeated); and the 2D Solve(qz, xv, yv) on a 32^2 field."""
    from waveletpotentials_b200 import fields
    out = {}
    for n in (8, 16):
        h = 1.0 / n
        s = shapes3((n, n, n))
        qx, qy, qz = (rng.standard_normal(s[k]) for k in ("qx", "qy", "qz"))
        qx[0] = qx[-1] = 0
        qx[:, :, 0] = qx[:, :, -1] = 0
        qy[0] = qy[-1] = 0
        qy[:, 0, :] = qy[:, -1, :] = 0
        qz[:, 0, :] = qz[:, -1, :] = 0
        qz[:, :, 0] = qz[:, :, -1] = 0
        xv, yv, zv = fields.curl3d(qx, qy, qz, (n, n, n), (h, h, h))
        res = run("psweep3d", {"xv": xv, "yv": yv, "zv": zv}, [n, h],
                  {"qx_solve": s["qx"], "qy_solve": s["qy"], "qz_solve": s["qz"], "qx": s["qx"], "qy": s["qy"],
                   "qz": s["qz"]})
        out[f"xv_{n}"], out[f"yv_{n}"], out[f"zv_{n}"] = xv, yv, zv
        for k, v in res.items():
            out[f"{k}_{n}"] = v
    n = 32
    h = 1.0 / n
    psi = rng.standard_normal((n + 1, n + 1))
    psi[0] = psi[-1] = 0
    psi[:, 0] = psi[:, -1] = 0
    xv2, yv2 = fields.curl2d(psi, (n, n), (h, h))
    out["qz2d"] = run("psweep2d", {"xv": xv2, "yv": yv2}, [n, h], {"qz": (n + 1, n + 1)})["qz"]
    out["xv2d"], out["yv2d"] = xv2, yv2
    save("psweep", **out)


def psweep_d_cases(rng):
    """CuParallelSweep3D with bc 'd': Solve alone (the z = 0 plane of qy from the x-integral of zv's
    bottom face, no top-plane step) on fields with wall flux, at 8^3 and 16^3; and the 2D Solve with
    bc 'd' (a y-integral of xv along x = 0, then the x-integral of yv) on a 32^2 field.  Project is
    not called: its bc 'd' branch (ProjectD) raised an illegal address at 16^3 in the first run of
    this recipe, so it is not run again."""
    from waveletpotentials_b200 import fields
    out = {}
    for n in (8, 16):
        h = 1.0 / n
        s = shapes3((n, n, n))
        qx, qy, qz = (rng.standard_normal(s[k]) for k in ("qx", "qy", "qz"))
        xv, yv, zv = fields.curl3d(qx, qy, qz, (n, n, n), (h, h, h))
        res = run("psweep3d", {"xv": xv, "yv": yv, "zv": zv}, [n, h, "d", 1],
                  {"qx_solve": s["qx"], "qy_solve": s["qy"], "qz_solve": s["qz"]})
        out[f"xv_{n}"], out[f"yv_{n}"], out[f"zv_{n}"] = xv, yv, zv
        for k, v in res.items():
            out[f"{k}_{n}"] = v
    n = 32
    h = 1.0 / n
    psi = rng.standard_normal((n + 1, n + 1))
    xv2, yv2 = fields.curl2d(psi, (n, n), (h, h))
    out["qz2d"] = run("psweep2d", {"xv": xv2, "yv": yv2}, [n, h, "d"], {"qz": (n + 1, n + 1)})["qz"]
    out["xv2d"], out["yv2d"] = xv2, yv2
    save("psweep_d", **out)


def psweep_mid_cases(rng):
    """CuParallelSweep3D::SolveFromMid (cuParallelSweep3D.cu:967-984): the z integrals of qx, qy run
    both ways from the plane mid.z, whose qy is the x-integral of zv both ways from mid.x; at 8^3 and
    16^3 with interior and zero mid indices, on fields with wall flux."""
    from waveletpotentials_b200 import fields
    out = {}
    for tag, n, mid in (("a8", 8, (4, 2, 3)), ("b16", 16, (7, 8, 11)), ("c8", 8, (0, 0, 0))):
        h = 1.0 / n
        s = shapes3((n, n, n))
        qx, qy, qz = (rng.standard_normal(s[k]) for k in ("qx", "qy", "qz"))
        xv, yv, zv = fields.curl3d(qx, qy, qz, (n, n, n), (h, h, h))
        res = run("psweep3d_mid", {"xv": xv, "yv": yv, "zv": zv}, [n, h, *mid],
                  {"qx": s["qx"], "qy": s["qy"], "qz": s["qz"]})
        out.update({f"{tag}_{k}": v for k, v in dict(xv=xv, yv=yv, zv=zv, **res).items()})
        out[f"{tag}_meta"] = np.array([n, *mid])
    save("psweep_mid", **out)


def domd_cases(rng):
    """CuDivLocalProject3D::ProjectLocal_q_ccc with the walls' boundary type 'd' (the base wavelet's bc
    proj_bc('d') = 'n', so cuProjectLocal_q_3d_nq_ccc runs) on random coefficients, and
    CuWaveletPotentialRecover3D::Solve with bc 'd' on random velocity fields with nonzero wall flux."""
    out = {}
    for tag, n3 in (("p16x8x32", (16, 8, 32)), ("p8", (8, 8, 8))):
        s = shapes3(n3)
        xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
        h = 1.0 / n3[0]
        r = run("project3d", {"xv": xv, "yv": yv, "zv": zv}, [*n3, h, "d"], {k: s[k] for k in ("qx", "qy", "qz")})
        out.update({f"{tag}_{k}": v for k, v in dict(xv=xv, yv=yv, zv=zv, **r).items()})
        out[f"{tag}_meta"] = np.array([*n3, h])
    for tag, n3 in (("r16", (16, 16, 16)), ("r8x16x32", (8, 16, 32))):
        s = shapes3(n3)
        xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
        h = 1.0 / n3[0]
        r = run("recover3d", {"xv": xv, "yv": yv, "zv": zv}, [*n3, h, "d"], {k: s[k] for k in ("qx", "qy", "qz")})
        out.update({f"{tag}_{k}": v for k, v in dict(xv=xv, yv=yv, zv=zv, **r).items()})
        out[f"{tag}_meta"] = np.array([*n3, h])
    save("domain_d", **out)


def domd2d_cases(rng):
    """The 2D counterparts with the walls' boundary type 'd': CuDivLocalProject::ProjectSingle with the
    base wavelet's bc proj_bc('d') = 'n' (cuProjectLocal_q_single_n runs) on random coefficients, and
    CuWaveletPotentialRecover2D::Solve with bc 'd' on random fields with nonzero wall flux; square,
    unequal-level (1, 2 and 5 levels apart: the three branches of GetDivL0Matrix the shapes reach)
    and unequal-spacing grids.  From the FP32 build: in the FP64 build cuProjectLocal_q_single_n needs
    72 registers a thread in its 1024-thread blocks, more than an SM holds, so its launch fails
    (cudaErrorLaunchOutOfResources) and the FP64 reference has no 2D Dirichlet-wall projection."""
    out = {}
    for tag, n2, hx, hy in (("p16", (16, 16), 1 / 16, 1 / 16), ("p32x16", (32, 16), 1 / 32, 1 / 16),
                            ("p16x64", (16, 64), 1 / 16, 1 / 64), ("p8x256", (8, 256), 1 / 8, 1 / 8)):
        xv, yv = rng.standard_normal((n2[0] + 1, n2[1])), rng.standard_normal((n2[0], n2[1] + 1))
        r = run("project2d", {"xv": xv, "yv": yv}, [*n2, hx, "d", hy], {"qz": (n2[0] + 1, n2[1] + 1)}, DRIVER32)
        assert np.any(r["qz"] != 0), tag
        out.update({f"{tag}_{k}": v for k, v in dict(xv=xv, yv=yv, **r).items()})
        out[f"{tag}_meta"] = np.array([*n2, hx, hy])
    for tag, n2, hx, hy in (("r16", (16, 16), 1 / 16, 1 / 16), ("r32x64", (32, 64), 1 / 32, 1 / 48),
                            ("r8x256", (8, 256), 1 / 8, 1 / 256)):
        xv, yv = rng.standard_normal((n2[0] + 1, n2[1])), rng.standard_normal((n2[0], n2[1] + 1))
        r = run("recover2d", {"xv": xv, "yv": yv}, [*n2, hx, "d", hy], {"qz": (n2[0] + 1, n2[1] + 1)}, DRIVER32)
        out.update({f"{tag}_{k}": v for k, v in dict(xv=xv, yv=yv, **r).items()})
        out[f"{tag}_meta"] = np.array([*n2, hx, hy])
    save("domain_d2d", **out)


def main():
    global OUT_DIR
    if "--out" in sys.argv:
        OUT_DIR = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(OUT_DIR, exist_ok=True)
    if not os.path.exists(DRIVER):
        sys.exit(f"{DRIVER} missing: run make -C oracle/refharness first (needs nvcc and the reference sources)")
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if only == "index":
        index_cases(np.random.default_rng(20261204))
        return
    if only == "cut":
        cut_cases(np.random.default_rng(20261205))
        return
    if only == "frac":
        frac_cases(np.random.default_rng(20261206))
        return
    if only == "sweep":
        sweep_cases(np.random.default_rng(20261207))
        return
    if only == "cdf35":
        cdf35_cases(np.random.default_rng(20261208))
        return
    if only == "dst":
        dst_cases(np.random.default_rng(20261209))
        return
    if only == "psweep":
        psweep_cases(np.random.default_rng(20261210))
        return
    if only == "domd":
        domd_cases(np.random.default_rng(20261211))
        return
    if only == "families":
        families_cases(np.random.default_rng(20261212))
        return
    if only == "short":
        short_cases(np.random.default_rng(20261213))
        return
    if only == "psweep_mid":
        psweep_mid_cases(np.random.default_rng(20261217))
        return
    if only == "psweep_d":
        psweep_d_cases(np.random.default_rng(20261216))
        return
    if only == "narrow":
        narrow_cases(np.random.default_rng(20261215))
        return
    if only == "domd2d":
        domd2d_cases(np.random.default_rng(20261214))
        return
    rng = np.random.default_rng(20261203)

    # 1D transforms along every axis, both wavelets, both boundary types, both directions
    dwt = {}
    for wav, ext in ((CDF3_7, 0), (CDF4_6, 1)):
        for bc in "nd":
            for fwd in (1, 0):
                for axis, (L, other) in {"y": (4, (3, 2)), "x": (5, (4, 3)), "z": (3, (5, 2))}.items():
                    n = (1 << L) + ext
                    if axis == "y":
                        DX, DY, DZ = other[0], n, other[1]
                    elif axis == "x":
                        DX, DY, DZ = n, other[0], other[1]
                    else:
                        DX, DY, DZ = other[0], other[1], n
                    a = rng.standard_normal((DZ, DX, DY))
                    out = run("dwt1d", {"a": a}, [DX, DY, DZ, L, axis, bc, wav, fwd], {"c": (DZ, DX, DY)})
                    key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_{axis}"
                    dwt[key + "_in"] = a
                    dwt[key + "_out"] = out["c"]
                    dwt[key + "_meta"] = np.array([DX, DY, DZ, L, ord(axis), ord(bc), wav, fwd])
    # long lines: the full 256-point y transform (the 256^3 line length)
    for wav, ext, bc in ((CDF3_7, 0, "n"), (CDF4_6, 1, "d")):
        for fwd in (1, 0):
            n = 256 + ext
            a = rng.standard_normal((1, 2, n))
            out = run("dwt1d", {"a": a}, [2, n, 1, 8, "y", bc, wav, fwd], {"c": (1, 2, n)})
            key = f"w{wav}_{bc}_{'f' if fwd else 'i'}_long"
            dwt[key + "_in"] = a
            dwt[key + "_out"] = out["c"]
            dwt[key + "_meta"] = np.array([2, n, 1, 8, ord("y"), ord(bc), wav, fwd])
    save("dwt1d", **dwt)

    # inner-product tables (8 bands of length dim; band 0 is the diagonal)
    ips = {}
    for n in (16, 32, 64):
        for wav, bc, dim in ((CDF3_7, "n", n), (CDF3_7, "d", n), (CDF4_6, "d", n + 1), (CDF4_6, "n", n + 1)):
            out = run("ip", {}, [dim, wav, bc], {"ip": (8, dim)})
            ips[f"ip_{dim}_{wav}_{bc}"] = out["ip"]
    save("ip_tables", **ips)

    # pointwise projections on random coefficient arrays
    n3 = (16, 8, 32)
    s = shapes3(n3)
    xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
    h = 1.0 / 16
    out = run("project3d", {"xv": xv, "yv": yv, "zv": zv}, [*n3, h], {k: s[k] for k in ("qx", "qy", "qz")})
    save("project3d", n=np.array(n3), h=h, xv=xv, yv=yv, zv=zv, **out)
    n2 = (32, 16)
    xv2, yv2 = rng.standard_normal((n2[0] + 1, n2[1])), rng.standard_normal((n2[0], n2[1] + 1))
    out = run("project2d", {"xv": xv2, "yv": yv2}, [*n2, 1.0 / 32], {"qz": (n2[0] + 1, n2[1] + 1)})
    save("project2d", n=np.array(n2), h=1.0 / 32, xv=xv2, yv=yv2, **out)

    # full potential recovery (random fields with zero wall-normal velocity)
    for tag, n3 in (("recover3d_16", (16, 16, 16)), ("recover3d_aniso", (8, 16, 32))):
        s = shapes3(n3)
        xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
        xv[:, 0, :] = xv[:, -1, :] = 0
        yv[:, :, 0] = yv[:, :, -1] = 0
        zv[0] = zv[-1] = 0
        h = 1.0 / n3[0]
        out = run("recover3d", {"xv": xv, "yv": yv, "zv": zv}, [*n3, h], {k: s[k] for k in ("qx", "qy", "qz")})
        save(tag, n=np.array(n3), h=h, xv=xv, yv=yv, zv=zv, **out)
    for tag, n2 in (("recover2d_32", (32, 32)), ("recover2d_aniso", (64, 16))):
        xv2, yv2 = rng.standard_normal((n2[0] + 1, n2[1])), rng.standard_normal((n2[0], n2[1] + 1))
        xv2[0] = xv2[-1] = 0
        yv2[:, 0] = yv2[:, -1] = 0
        h = 1.0 / n2[0]
        out = run("recover2d", {"xv": xv2, "yv": yv2}, [*n2, h], {"qz": (n2[0] + 1, n2[1] + 1)})
        save(tag, n=np.array(n2), h=h, xv=xv2, yv=yv2, **out)

    # solid fractions from a sphere level set (TestLocalProjection.cpp:621-627 geometry)
    fr = {}
    for n, r in ((16, 0.245), (32, 0.2)):
        h = 1.0 / n
        out = run("frac3d", {}, [n, h, 0.5, 0.5, 0.5, r], {k: shapes3((n, n, n))[k2] for k, k2 in
                                                           (("ax", "xv"), ("ay", "yv"), ("az", "zv"))})
        for k, v in out.items():
            fr[f"{k}_{n}"] = v
        fr[f"r_{n}"] = np.array(r)
    save("fractions3d", **fr)

    # divergence and gradient update with fractions
    n = 16
    s = shapes3((n, n, n))
    ax, ay, az = fr["ax_16"], fr["ay_16"], fr["az_16"]
    xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
    p = rng.standard_normal(s["p"])
    out = run("div3d", {"xv": xv, "yv": yv, "zv": zv, "ax": ax, "ay": ay, "az": az}, [n, n, n, 1.0 / n],
              {"b": s["p"]})
    out2 = run("grad3d", {"xv": xv, "yv": yv, "zv": zv, "ax": ax, "ay": ay, "az": az, "p": p}, [n, n, n, 1.0 / n],
               {"xv": s["xv"], "yv": s["yv"], "zv": s["zv"]})
    save("divgrad3d", n=np.array([n, n, n]), h=1.0 / n, xv=xv, yv=yv, zv=zv, p=p, ax=ax, ay=ay, az=az, b=out["b"],
         xv_out=out2["xv"], yv_out=out2["yv"], zv_out=out2["zv"])

    # fractional multigrid: per-cycle residual history and the solution
    for tag, n, frs, cyc, nu, w in (("mg3d_16", 16, "16", 6, (2, 2), 2.0 / 3.0), ("mg3d_32", 32, "32", 4, (3, 3), 0.8)):
        s = shapes3((n, n, n))
        ax, ay, az = fr["ax_" + frs], fr["ay_" + frs], fr["az_" + frs]
        xv, yv, zv = (rng.standard_normal(s[k]) for k in ("xv", "yv", "zv"))
        xv[:, 0, :] = xv[:, -1, :] = 0
        yv[:, :, 0] = yv[:, :, -1] = 0
        zv[0] = zv[-1] = 0
        f = run("div3d", {"xv": xv, "yv": yv, "zv": zv, "ax": ax, "ay": ay, "az": az}, [n, n, n, 1.0 / n],
                {"b": s["p"]})["b"]
        out = run("mg3d", {"f": f, "ax": ax, "ay": ay, "az": az}, [n, n, n, 1.0 / n, cyc, nu[0], nu[1], w],
                  {"p": s["p"], "hist": (cyc,)})
        save(tag, n=np.array([n, n, n]), h=1.0 / n, f=f, ax=ax, ay=ay, az=az, ncycles=cyc, nu=np.array(nu), omega=w,
             **out)
    n2 = (32, 32)
    ax2 = np.clip(rng.uniform(-0.3, 1.3, (n2[0] + 1, n2[1])), 0, 1)
    ay2 = np.clip(rng.uniform(-0.3, 1.3, (n2[0], n2[1] + 1)), 0, 1)
    f2 = rng.standard_normal(n2)
    f2 -= f2.mean()
    out = run("mg2d", {"f": f2, "ax": ax2, "ay": ay2}, [*n2, 1.0 / 32, 5, 5, 5, 0.8], {"p": n2, "hist": (5,)})
    save("mg2d_32", n=np.array(n2), h=1.0 / 32, f=f2, ax=ax2, ay=ay2, ncycles=5, nu=np.array([5, 5]), omega=0.8, **out)
    index_cases(np.random.default_rng(20261204))
    cut_cases(np.random.default_rng(20261205))
    frac_cases(np.random.default_rng(20261206))
    sweep_cases(np.random.default_rng(20261207))
    cdf35_cases(np.random.default_rng(20261208))


if __name__ == "__main__":
    main()
