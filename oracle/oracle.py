"""FP64 CPU oracle of the WaveletPotentials projection-and-recovery path (ctypes wrapper).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it as the checker; the product package never
imports it.  The arithmetic lives in ``wp_oracle.c`` (a plain-C restatement of the reference
algorithm, each routine citing the reference file:line it follows).

Arrays use the reference layout (``Utils.h:46-47``): a 3D array with extents (DX, DY, DZ) is a
numpy array of shape (DZ, DX, DY), so y is the fastest index; 2D arrays are (DX, DY).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwp_oracle.so")
CDF4_6 = 7
CDF3_7 = 11

_lib = None


def build(force: bool = False) -> str:
    """Compile wp_oracle.c into libwp_oracle.so (gcc, OpenMP)."""
    src = os.path.join(HERE, "wp_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-std=gnu11", "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        d = ctypes.c_double
        i = ctypes.c_int
        p = ctypes.c_void_p
        c = ctypes.c_char
        sig = {
            "or_dwt_line": (i, [p, i, i, i, c, i]),
            "or_dwt_axis": (i, [p, i, i, i, i, c, i, c, i]),
            "or_ip_diag": (i, [p, i, i, c]),
            "or_project3d": (i, [p, p, p, p, p, p, i, i, i, d, d, d]),
            "or_project3d_nq": (i, [p, p, p, p, p, p, i, i, i, d, d, d]),
            "or_project2d": (i, [p, p, p, i, i, d, d]),
            "or_project2d_nq": (i, [p, p, p, i, i, d, d]),
            "or_recover3d": (i, [p, p, p, p, p, p, i, i, i, d, d, d, c]),
            "or_recover2d": (i, [p, p, p, i, i, d, d, c]),
            "or_curl3d": (None, [p, p, p, p, p, p, i, i, i, d, d, d]),
            "or_curl2d": (None, [p, p, p, i, i, d, d]),
            "or_divergence3d": (None, [p, p, p, p, p, p, p, i, i, i, d, d, d]),
            "or_divergence2d": (None, [p, p, p, p, p, i, i, d, d]),
            "or_grad_subtract3d": (None, [p, p, p, p, p, p, p, i, i, i, d, d, d, i]),
            "or_grad_subtract2d": (None, [p, p, p, p, p, i, i, d, d, i]),
            "or_sdf_spheres3d": (None, [p, i, i, i, d, p, p, i]),
            "or_sdf_boxes3d": (None, [p, i, i, i, d, p, p, i]),
            "or_fractions3d": (None, [p, p, p, p, i, i, i, d]),
            "or_fractions2d": (None, [p, p, p, i, i, d]),
            "or_mgfrac3d_solve": (i, [p, p, p, p, p, p, i, i, i, d, d, d, i, i, i, d, i, p]),
            "or_mgfrac3d_solve_index": (i, [p, p, p, p, p, p, i, i, i, d, d, d, i, i, i, d, p, p]),
            "or_cut3d": (i, [p, p, p, i, i, i, i]),
            "or_fast_sweep": (None, [p, i, i, i, d, i, i]),
            "or_particles_to_ls": (None, [p, p, i, i, i, i, d, d, d, i]),
            "or_particles_to_ls_narrow": (None, [p, p, i, i, i, i, d, d, i]),
            "or_fractions3d_subsampled": (None, [p, p, p, p, i, i, i, d]),
            "or_mgfrac2d_solve": (i, [p, p, p, p, p, i, i, d, d, i, i, i, d, i, p]),
            "or_frac_residual3d": (d, [p, p, p, p, p, p, i, i, i, d, d, d]),
            "or_frac_residual2d": (d, [p, p, p, p, p, i, i, d, d]),
            "or_dst3d_poisson": (None, [p, p, i, i, i, d, d, d]),
            "or_set_threads": (None, [i]),
            "or_get_threads": (i, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def set_threads(n: int) -> None:
    """OpenMP threads of the oracle's parallel loops."""
    lib().or_set_threads(int(n))


def threads() -> int:
    """OpenMP threads the oracle's parallel loops use."""
    return int(lib().or_get_threads())


def _p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with code {rc}")


# ---------------------------------------------------------------- transforms
def dwt_line(line, levels: int, wavelet: int, bc: str, forward: bool) -> np.ndarray:
    out = _f64(line).copy()
    _check(lib().or_dwt_line(_p(out), out.size, levels, wavelet, bc.encode(), int(forward)), "dwt_line")
    return out


def dwt_axis(arr, levels: int, axis: str, wavelet: int, bc: str, forward: bool) -> np.ndarray:
    """arr: 3D array of shape (DZ, DX, DY) or 2D (DX, DY)."""
    a = _f64(arr).copy()
    shp = a.shape if a.ndim == 3 else (1,) + a.shape
    dz, dx, dy = shp
    _check(lib().or_dwt_axis(_p(a), dx, dy, dz, levels, axis.encode(), wavelet, bc.encode(), int(forward)),
           "dwt_axis")
    return a


def ip_diag(dim: int, wavelet: int, bc: str) -> np.ndarray:
    out = np.zeros(dim)
    _check(lib().or_ip_diag(_p(out), dim, wavelet, bc.encode()), "ip_diag")
    return out


# ------------------------------------------------------------- shapes helpers
def mac_shapes3d(nx, ny, nz):
    return {"xv": (nz, nx + 1, ny), "yv": (nz, nx, ny + 1), "zv": (nz + 1, nx, ny),
            "qx": (nz + 1, nx, ny + 1), "qy": (nz + 1, nx + 1, ny), "qz": (nz, nx + 1, ny + 1),
            "p": (nz, nx, ny)}


def mac_shapes2d(nx, ny):
    return {"xv": (nx + 1, ny), "yv": (nx, ny + 1), "qz": (nx + 1, ny + 1), "p": (nx, ny)}


# ----------------------------------------------------------------- projection
def project3d(xv, yv, zv, n, d, bc="n"):
    """The local projection of the recovery; bc: the walls' boundary type ('n': cuProjectLocal_q_3d_dq_ccc,
    'd': cuProjectLocal_q_3d_nq_ccc)."""
    nx, ny, nz = n
    s = mac_shapes3d(nx, ny, nz)
    qx, qy, qz = (np.zeros(s[k]) for k in ("qx", "qy", "qz"))
    fn = lib().or_project3d if bc == "n" else lib().or_project3d_nq
    _check(fn(_p(qx), _p(qy), _p(qz), _p(_f64(xv)), _p(_f64(yv)), _p(_f64(zv)), nx, ny, nz, *d), "project3d")
    return qx, qy, qz


def project2d(xv, yv, n, d, bc="n"):
    """CuDivLocalProject::ProjectSingle for the walls' boundary type bc ('n': cuProjectLocal_q_single,
    'd': cuProjectLocal_q_single_n)."""
    nx, ny = n
    qz = np.zeros((nx + 1, ny + 1))
    fn = lib().or_project2d if bc == "n" else lib().or_project2d_nq
    _check(fn(_p(qz), _p(_f64(xv)), _p(_f64(yv)), nx, ny, *d), "project2d")
    return qz


def recover3d(xv, yv, zv, n, d, bc="n"):
    nx, ny, nz = n
    s = mac_shapes3d(nx, ny, nz)
    qx, qy, qz = (np.zeros(s[k]) for k in ("qx", "qy", "qz"))
    _check(lib().or_recover3d(_p(qx), _p(qy), _p(qz), _p(_f64(xv)), _p(_f64(yv)), _p(_f64(zv)), nx, ny, nz, *d,
                              bc.encode()), "recover3d")
    return qx, qy, qz


def recover2d(xv, yv, n, d, bc="n"):
    nx, ny = n
    qz = np.zeros((nx + 1, ny + 1))
    _check(lib().or_recover2d(_p(qz), _p(_f64(xv)), _p(_f64(yv)), nx, ny, *d, bc.encode()), "recover2d")
    return qz


def cut3d(qx, qy, qz, n, level):
    """CuWaveletPotentialRecover3D::CutCoefficients: the potential with its wavelet coefficients
    below `level` cleared (returns new arrays)."""
    out = [np.array(_f64(a)) for a in (qx, qy, qz)]
    _check(lib().or_cut3d(*(_p(a) for a in out), *n, level), "or_cut3d")
    return tuple(out)


def curl3d(qx, qy, qz, n, d):
    nx, ny, nz = n
    s = mac_shapes3d(nx, ny, nz)
    xv, yv, zv = (np.zeros(s[k]) for k in ("xv", "yv", "zv"))
    lib().or_curl3d(_p(xv), _p(yv), _p(zv), _p(_f64(qx)), _p(_f64(qy)), _p(_f64(qz)), nx, ny, nz, *d)
    return xv, yv, zv


def curl2d(qz, n, d):
    nx, ny = n
    xv, yv = np.zeros((nx + 1, ny)), np.zeros((nx, ny + 1))
    lib().or_curl2d(_p(xv), _p(yv), _p(_f64(qz)), nx, ny, *d)
    return xv, yv


# -------------------------------------------------------- divergence / gradient
def divergence3d(xv, yv, zv, ax, ay, az, n, d):
    nx, ny, nz = n
    b = np.zeros((nz, nx, ny))
    lib().or_divergence3d(_p(b), _p(_f64(xv)), _p(_f64(yv)), _p(_f64(zv)), _p(_f64(ax)), _p(_f64(ay)),
                          _p(_f64(az)), nx, ny, nz, *d)
    return b


def divergence2d(xv, yv, ax, ay, n, d):
    nx, ny = n
    b = np.zeros((nx, ny))
    lib().or_divergence2d(_p(b), _p(_f64(xv)), _p(_f64(yv)), _p(_f64(ax)), _p(_f64(ay)), nx, ny, *d)
    return b


def grad_subtract3d(xv, yv, zv, p, ax, ay, az, n, d, multiply_frac=True):
    nx, ny, nz = n
    xo, yo, zo = _f64(xv).copy(), _f64(yv).copy(), _f64(zv).copy()
    lib().or_grad_subtract3d(_p(xo), _p(yo), _p(zo), _p(_f64(p)), _p(_f64(ax)), _p(_f64(ay)), _p(_f64(az)),
                             nx, ny, nz, *d, int(multiply_frac))
    return xo, yo, zo


def grad_subtract2d(xv, yv, p, ax, ay, n, d, multiply_frac=True):
    nx, ny = n
    xo, yo = _f64(xv).copy(), _f64(yv).copy()
    lib().or_grad_subtract2d(_p(xo), _p(yo), _p(_f64(p)), _p(_f64(ax)), _p(_f64(ay)), nx, ny, *d,
                             int(multiply_frac))
    return xo, yo


# --------------------------------------------------------------------- solids
def sdf_spheres3d(n, dx, centers, radii):
    nx, ny, nz = n
    sdf = np.zeros((nz, nx, ny))
    c = _f64(np.reshape(centers, (-1, 3)))
    r = _f64(np.reshape(radii, (-1,)))
    lib().or_sdf_spheres3d(_p(sdf), nx, ny, nz, dx, _p(c), _p(r), r.size)
    return sdf


def sdf_boxes3d(sdf, n, dx, lo, hi):
    nx, ny, nz = n
    out = _f64(sdf).copy()
    lo_, hi_ = _f64(np.reshape(lo, (-1, 3))), _f64(np.reshape(hi, (-1, 3)))
    lib().or_sdf_boxes3d(_p(out), nx, ny, nz, dx, _p(lo_), _p(hi_), lo_.shape[0])
    return out


def fractions3d(sdf, n, dx):
    nx, ny, nz = n
    s = mac_shapes3d(nx, ny, nz)
    ax, ay, az = (np.zeros(s[k]) for k in ("xv", "yv", "zv"))
    lib().or_fractions3d(_p(ax), _p(ay), _p(az), _p(_f64(sdf)), nx, ny, nz, dx)
    return ax, ay, az


def fractions3d_subsampled(ls, n, dx):
    """CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx): cut faces sub-sampled 128 x 128."""
    nx, ny, nz = n
    s = mac_shapes3d(nx, ny, nz)
    ax, ay, az = (np.zeros(s[k]) for k in ("xv", "yv", "zv"))
    lib().or_fractions3d_subsampled(_p(ax), _p(ay), _p(az), _p(_f64(ls)), nx, ny, nz, dx)
    return ax, ay, az


def fast_sweep(ls, n, dx, iters, reinit=False):
    """CuFastSweeping::Solve (reinit=False) / ReinitLevelSet (True) as Jacobi iterations."""
    out = np.array(_f64(ls))
    lib().or_fast_sweep(_p(out), *n, dx, iters, int(bool(reinit)))
    return out


def particles_to_ls(xyz, n, dx, radius, max_dis, iters):
    """CuFastSweeping::ParticlesToLs; xyz (count, 3) positions; returns the level set (DZ, DX, DY)."""
    nx, ny, nz = n
    out = np.zeros((nz, nx, ny))
    pts = _f64(np.reshape(xyz, (-1, 3)))
    lib().or_particles_to_ls(_p(out), _p(pts), pts.shape[0], nx, ny, nz, dx, radius, max_dis, iters)
    return out


def particles_to_ls_narrow(ls, xyz, n, dx, radius, iters):
    """CuFastSweeping::ParticlesToLsNarrow; ls (DZ, DX, DY) is the start; returns the new level set."""
    out = np.array(_f64(ls))
    pts = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    nx, ny, nz = n
    lib().or_particles_to_ls_narrow(_p(out), _p(pts), pts.shape[0], nx, ny, nz, dx, radius, iters)
    return out


def fractions2d(sdf, n, dx):
    nx, ny = n
    ax, ay = np.zeros((nx + 1, ny)), np.zeros((nx, ny + 1))
    lib().or_fractions2d(_p(ax), _p(ay), _p(_f64(sdf)), nx, ny, dx)
    return ax, ay


# ------------------------------------------------------------------ multigrid
PROLONG_CONSTANT = 0   # the reference's V-cycle
PROLONG_TRILINEAR = 1  # convergent variant


def mgfrac3d_solve(f, ax, ay, az, n, d, ncycles, nu1, nu2, omega, p0=None, prolong=PROLONG_CONSTANT):
    nx, ny, nz = n
    p = np.zeros((nz, nx, ny))
    hist = np.zeros(max(ncycles, 1))
    lib().or_mgfrac3d_solve(_p(p), _p(None if p0 is None else _f64(p0)), _p(_f64(f)), _p(_f64(ax)),
                            _p(_f64(ay)), _p(_f64(az)), nx, ny, nz, *d, ncycles, nu1, nu2, omega, prolong,
                            _p(hist))
    return p, hist[:ncycles]


def mgfrac3d_solve_index(f, ax, ay, az, n, d, ncycles, nu1, nu2, omega, p0=None):
    """Index-sparse V-cycles (CuMultigridFrac3D::Solve_index); returns (p, history, listed cells per level)."""
    nx, ny, nz = n
    p = np.zeros((nz, nx, ny))
    hist = np.zeros(max(ncycles, 1))
    counts = np.zeros(32, dtype=np.int64)
    nl = lib().or_mgfrac3d_solve_index(_p(p), _p(None if p0 is None else _f64(p0)), _p(_f64(f)), _p(_f64(ax)),
                                       _p(_f64(ay)), _p(_f64(az)), nx, ny, nz, *d, ncycles, nu1, nu2, omega,
                                       _p(hist), counts.ctypes.data_as(ctypes.c_void_p))
    return p, hist[:ncycles], counts[:nl].copy()


def mgfrac2d_solve(f, ax, ay, n, d, ncycles, nu1, nu2, omega, p0=None, prolong=PROLONG_CONSTANT):
    nx, ny = n
    p = np.zeros((nx, ny))
    hist = np.zeros(max(ncycles, 1))
    lib().or_mgfrac2d_solve(_p(p), _p(None if p0 is None else _f64(p0)), _p(_f64(f)), _p(_f64(ax)),
                            _p(_f64(ay)), nx, ny, *d, ncycles, nu1, nu2, omega, prolong, _p(hist))
    return p, hist[:ncycles]


def frac_residual3d(p, f, ax, ay, az, n, d):
    nx, ny, nz = n
    r = np.zeros((nz, nx, ny))
    rel = lib().or_frac_residual3d(_p(r), _p(_f64(p)), _p(_f64(f)), _p(_f64(ax)), _p(_f64(ay)), _p(_f64(az)),
                                   nx, ny, nz, *d)
    return rel, r


def frac_residual2d(p, f, ax, ay, n, d):
    nx, ny = n
    r = np.zeros((nx, ny))
    rel = lib().or_frac_residual2d(_p(r), _p(_f64(p)), _p(_f64(f)), _p(_f64(ax)), _p(_f64(ay)), nx, ny, *d)
    return rel, r


def dst3d_poisson(f, n, d):
    nx, ny, nz = n
    p = np.zeros((nz, nx, ny))
    lib().or_dst3d_poisson(_p(p), _p(_f64(f)), nx, ny, nz, *d)
    return p


# ------------------------------------------------------------ sweep + DST recovery
def sweep3d_solve(xv, yv, zv, n, d, bc="n"):
    """CuParallelSweep3D::Solve (cuParallelSweep3D.cu:939-966): qz = 0; qx, qy start from their z = 0
    plane and integrate yv (+dz) and xv (-dz) along z (SweepingQx / SweepingQy, :28-66).  bc 'n': the
    z = 0 planes are 0 and the top plane is then made tangential-free: qp = the x-integral of qx's top
    plane (cuSweepingQ_x, :9-26), qx and qy top planes cleared, qz's top plane gets -qp / dz
    (CudaMatAdd, cudaMath.cu:110-118).  bc 'd' (SetQxQyBoundary, :925-937): qx's z = 0 plane is 0 and
    qy's is the x-integral of zv's bottom face (SweepingQy_x, :68-85), with no top-plane step.  FP64
    sums in the reference's sequential order."""
    nx, ny, nz = n
    dx, dy, dz = d
    xv, yv = _f64(xv), _f64(yv)
    s = mac_shapes3d(nx, ny, nz)
    qx, qy, qz = (np.zeros(s[k]) for k in ("qx", "qy", "qz"))
    if bc == "d":
        zv = _f64(zv)
        for x in range(1, nx + 1):
            qy[0, x] = qy[0, x - 1] + zv[0, x - 1] * dx
    for z in range(1, nz + 1):
        qx[z] = qx[z - 1] + yv[z - 1] * dz
        qy[z] = qy[z - 1] - xv[z - 1] * dz
    if bc == "d":
        return qx, qy, qz
    qp = np.zeros((nx + 1, ny + 1))
    for x in range(1, nx + 1):
        qp[x] = qp[x - 1] + qx[nz, x - 1] * dx
    qx[nz] = 0.0
    qy[nz] = 0.0
    qz[nz - 1] += qp * (-1.0 / dz)
    return qx, qy, qz


def sweep3d_solve_from_mid(xv, yv, zv, n, d, mid):
    """CuParallelSweep3D::SolveFromMid (cuParallelSweep3D.cu:967-984; SweepingQy_x_mid, SweepingQx_mid,
    SweepingQy_mid, :145-214): qz = 0; qx's plane mid.z is 0; qy's plane mid.z is the x-integral of
    zv's plane mid.z both ways from 0 at x = mid.x (the reference leaves that row as the caller's
    buffer had it); then qx, qy integrate yv (+dz), xv (-dz) along z both ways from plane mid.z.
    mid.y is not used.  FP64 sums in the reference's sequential order."""
    nx, ny, nz = n
    dx, dy, dz = d
    mx, _, mz = mid
    xv, yv, zv = _f64(xv), _f64(yv), _f64(zv)
    s = mac_shapes3d(nx, ny, nz)
    qx, qy, qz = (np.zeros(s[k]) for k in ("qx", "qy", "qz"))
    for x in range(mx - 1, -1, -1):
        qy[mz, x] = qy[mz, x + 1] - zv[mz, x] * dx
    for x in range(mx + 1, nx + 1):
        qy[mz, x] = qy[mz, x - 1] + zv[mz, x - 1] * dx
    for z in range(mz - 1, -1, -1):
        qx[z] = qx[z + 1] - yv[z] * dz
        qy[z] = qy[z + 1] + xv[z] * dz
    for z in range(mz + 1, nz + 1):
        qx[z] = qx[z - 1] + yv[z - 1] * dz
        qy[z] = qy[z - 1] - xv[z - 1] * dz
    return qx, qy, qz


def sweep3d_project(qx, qy, qz, n, d):
    """CuParallelSweep3D::ProjectZero (cuParallelSweep3D.cu:1043-1081): b = -div q on the (n-1)^3
    interior nodes (cuGetB_q_zero_3d, cuConvergence.cu:126-159), the DST-I Poisson solve on them,
    q -= grad phi with phi = 0 on the boundary nodes (cuGradientMinus3D_zero_Q, cuGradient.cu:2353-2405,
    including its choice of spacing for the three wall edges)."""
    nx, ny, nz = n
    dxi, dyi, dzi = (1.0 / v for v in d)
    qx, qy, qz = (_f64(a).copy() for a in (qx, qy, qz))
    b = -((qx[1:nz, 1:nx, 1:ny] - qx[1:nz, 0:nx - 1, 1:ny]) * dxi +
          (qy[1:nz, 1:nx, 1:ny] - qy[1:nz, 1:nx, 0:ny - 1]) * dyi +
          (qz[1:nz, 1:nx, 1:ny] - qz[0:nz - 1, 1:nx, 1:ny]) * dzi)
    P = dst3d_poisson(b, (nx - 1, ny - 1, nz - 1), d)
    qy[1:nz, 1:nx, 0] -= P[:, :, 0] * dxi
    qx[1:nz, 0, 1:ny] -= P[:, 0, :] * dyi
    qz[0, 1:nx, 1:ny] -= P[0, :, :] * dzi
    gy = -P * dyi
    gy[:, :, :-1] += P[:, :, 1:] * dyi
    gx = -P * dxi
    gx[:, :-1, :] += P[:, 1:, :] * dxi
    gz = -P * dzi
    gz[:-1] += P[1:] * dzi
    qy[1:nz, 1:nx, 1:ny] -= gy
    qx[1:nz, 1:nx, 1:ny] -= gx
    qz[1:nz, 1:nx, 1:ny] -= gz
    return qx, qy, qz


def sweep2d_solve(yv, n, d, bc="n", xv=None):
    """CuParallelSweep3D::Solve(qz, xv, yv) (cuParallelSweep3D.cu:986-998): bc 'n' (SweepingQz_x_0,
    :106-124): qz = 0 on x = 0, qz[x] = qz[x-1] - yv[x-1] dx.  bc 'd' (SweepingQz_y, :126-143, then
    SweepingQz_x, :87-104): the x = 0 column is the y-integral of xv's x = 0 column from qz(0, 0) =
    0 (the reference leaves that entry as the caller's buffer had it), then the same x-integral."""
    nx, ny = n
    yv = _f64(yv)
    qz = np.zeros((nx + 1, ny + 1))
    if bc == "d":
        xv = _f64(xv)
        for y in range(1, ny + 1):
            qz[0, y] = qz[0, y - 1] + xv[0, y - 1] * d[1]
    for x in range(1, nx + 1):
        qz[x] = qz[x - 1] - yv[x - 1] * d[0]
    return qz


# -------------------------------------------------------------------- metrics
def rel_l2(ref, got) -> float:
    """Relative L2 error, CalculateErrorL2 (Utils.cpp:184-210): sqrt(sum (a-b)^2 / sum a^2)."""
    ref = np.asarray(ref, dtype=np.float64)
    got = np.asarray(got, dtype=np.float64)
    den = float(np.sum(ref * ref))
    return float(np.sqrt(np.sum((ref - got) ** 2) / den)) if den > 0 else float(np.sqrt(np.sum(got * got)))


def rel_l2_multi(refs, gots) -> float:
    num = sum(float(np.sum((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2)) for a, b in zip(refs, gots))
    den = sum(float(np.sum(np.asarray(a, np.float64) ** 2)) for a in refs)
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))


# ----------------------------------------------------------------------------- warm-start network
# FP64 restatement of the 3x3x3 zero-padded convolution of the warm-start network (no reference
# counterpart).  Volumes are channels-last (nz, nx, ny, c); weights (27, cout, cin) with
# tap = (dz*3 + dx)*3 + dy for offsets (dz-1, dx-1, dy-1).

def bf16_round(a) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _shifted(x, dz, dx, dy):
    """x[z+dz-1, x+dx-1, y+dy-1] with zeros outside (x is (nz, nx, ny, c))."""
    p = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    nz, nx, ny = x.shape[:3]
    return p[dz:dz + nz, dx:dx + nx, dy:dy + ny]


def conv3d_forward(x, w, bias=None):
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    out = np.zeros(x.shape[:3] + (w.shape[1],))
    for t in range(27):
        dz, dx, dy = t // 9, (t // 3) % 3, t % 3
        out += np.einsum("zxyc,oc->zxyo", _shifted(x, dz, dx, dy), w[t])
    if bias is not None:
        out += np.asarray(bias, np.float64)
    return out


def conv3d_input_grad(gy, w):
    """d/dx of sum(gy * conv3d_forward(x, w)): the convolution with flipped, transposed weights."""
    wt = np.transpose(np.asarray(w, np.float64)[::-1], (0, 2, 1))
    return conv3d_forward(gy, wt)


def conv3d_weight_grad(x, gy):
    x = np.asarray(x, np.float64)
    gy = np.asarray(gy, np.float64)
    dw = np.zeros((27, gy.shape[3], x.shape[3]))
    for t in range(27):
        dz, dx, dy = t // 9, (t // 3) % 3, t % 3
        dw[t] = np.einsum("zxyo,zxyc->oc", gy, _shifted(x, dz, dx, dy))
    return dw


# The warm-start U-Net in FP64 (same architecture, parameter order and loss as wp_unet.cu).
UNET_SPEC = [(16, 0, 16), (16, 0, 16), (16, 0, 32), (32, 0, 32), (32, 0, 64), (64, 0, 64), (32, 64, 32),
             (32, 0, 32), (16, 32, 16), (16, 0, 16)]


def unet_unflatten(vec):
    vec = np.asarray(vec, np.float64)
    convs, off = [], 0
    for cin0, cin1, cout in UNET_SPEC:
        ws = []
        for cin in (cin0, cin1):
            if cin:
                n = 27 * cout * cin
                ws.append(vec[off:off + n].reshape(27, cout, cin))
                off += n
        b = vec[off:off + cout]
        off += cout
        convs.append((ws, b))
    head = vec[off:off + 17]
    assert off + 17 == vec.size
    return convs, head


def unet_flatten(convs, head):
    parts = []
    for ws, b in convs:
        parts += [w.ravel() for w in ws] + [np.ravel(b)]
    parts.append(np.ravel(head))
    return np.concatenate(parts)


def _pool(x):
    nz, nx, ny, c = x.shape
    return x.reshape(nz // 2, 2, nx // 2, 2, ny // 2, 2, c).mean(axis=(1, 3, 5))


def _up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=0), 2, axis=1), 2, axis=2)


def _up_bwd(g):
    nz, nx, ny, c = g.shape
    return g.reshape(nz // 2, 2, nx // 2, 2, ny // 2, 2, c).sum(axis=(1, 3, 5))


def unet_forward(vec, b, sdf, hcell, bf16=False):
    """Returns (p prediction in physical units, cache).  b, sdf: (nz, nx, ny).  The network works on
    p * tscale / rms(b) with tscale = 4 pi^2 / Lx^2 (Lx = nx h).  bf16=True rounds the weights and
    every stored activation to BF16 where the GPU network stores them (the arithmetic stays FP64)."""
    convs, head = unet_unflatten(vec)
    R = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    if bf16:
        convs = [([R(w) for w in ws], bb) for ws, bb in convs]
    b = np.asarray(b, np.float64)
    rms = np.sqrt(np.mean(b * b))
    x = np.zeros(b.shape + (16,))
    x[..., 0] = b / rms if rms > 0 else 0.0
    x[..., 1] = np.clip(np.asarray(sdf, np.float64) / (4.0 * hcell), -1.0, 1.0)
    x = R(x)
    relu = lambda v: np.maximum(v, 0.0)
    def conv(i, *xs):
        ws, bb = convs[i]
        return R(relu(sum(conv3d_forward(xx, w) for xx, w in zip(xs, ws)) + bb))
    c = {"in": x, "R": R, "convs": convs}
    c["a1"] = conv(0, x)
    c["s1"] = conv(1, c["a1"])
    c["p1"] = R(_pool(c["s1"]))
    c["a2"] = conv(2, c["p1"])
    c["s2"] = conv(3, c["a2"])
    c["p2"] = R(_pool(c["s2"]))
    c["a3"] = conv(4, c["p2"])
    c["e3"] = conv(5, c["a3"])
    c["u2"] = _up(c["e3"])
    c["a4"] = conv(6, c["s2"], c["u2"])
    c["e2"] = conv(7, c["a4"])
    c["u1"] = _up(c["e2"])
    c["a5"] = conv(8, c["s1"], c["u1"])
    c["e1"] = conv(9, c["a5"])
    c["pred"] = c["e1"] @ head[:16] + head[16]
    c["rms"] = rms
    c["tscale"] = 4.0 * np.pi ** 2 / (b.shape[1] * hcell) ** 2  # 4 pi^2 / Lx^2, Lx = nx h
    return c["pred"] * rms / c["tscale"], c


def unet_loss_grad(vec, b, sdf, p, hcell, bf16=False):
    """Loss of wp_unet_train_step and its gradient (flattened in the parameter order); bf16=True
    also rounds the stored gradients to BF16 where the GPU network stores them."""
    _, head = unet_unflatten(vec)
    _, c = unet_forward(vec, b, sdf, hcell, bf16)
    convs, R = c["convs"], c["R"]
    fluid = np.asarray(sdf) > 0
    r = c["pred"] - np.asarray(p, np.float64) * c["tscale"] / c["rms"]
    cnt = max(int(fluid.sum()), 1)
    mu = r[fluid].sum() / cnt
    rr = np.where(fluid, r - mu, 0.0)
    loss = float(np.sum(rr * rr) / cnt)
    g = 2.0 * rr / cnt
    gconv = [[None for _ in ws] for ws, _ in convs]
    gbias = [None] * len(convs)
    ghead = np.concatenate([np.einsum("zxy,zxyc->c", g, c["e1"]), [g.sum()]])
    mask = lambda gy, y: np.where(y > 0, gy, 0.0)

    def back(i, gy, xs, need):
        """gy: gradient wrt the (post-ReLU masked) pre-activation; returns input grads of each part."""
        ws, _ = convs[i]
        gbias[i] = gy.sum(axis=(0, 1, 2))
        outs = []
        for k, (xx, w) in enumerate(zip(xs, ws)):
            gconv[i][k] = conv3d_weight_grad(xx, gy)
            outs.append(conv3d_input_grad(gy, w) if need else None)
        return outs
    g_e1 = R(mask(g[..., None] * head[:16], c["e1"]))
    g_a5 = R(mask(back(9, g_e1, [c["a5"]], True)[0], c["a5"]))
    g_s1p, g_u1 = (R(t) for t in back(8, g_a5, [c["s1"], c["u1"]], True))
    g_e2 = R(mask(_up_bwd(g_u1), c["e2"]))
    g_a4 = R(mask(back(7, g_e2, [c["a4"]], True)[0], c["a4"]))
    g_s2p, g_u2 = (R(t) for t in back(6, g_a4, [c["s2"], c["u2"]], True))
    g_e3 = R(mask(_up_bwd(g_u2), c["e3"]))
    g_a3 = R(mask(back(5, g_e3, [c["a3"]], True)[0], c["a3"]))
    g_p2 = R(back(4, g_a3, [c["p2"]], True)[0])
    g_s2 = R(mask(g_s2p + _up(g_p2) / 8.0, c["s2"]))
    g_a2 = R(mask(back(3, g_s2, [c["a2"]], True)[0], c["a2"]))
    g_p1 = R(back(2, g_a2, [c["p1"]], True)[0])
    g_s1 = R(mask(g_s1p + _up(g_p1) / 8.0, c["s1"]))
    g_a1 = R(mask(back(1, g_s1, [c["a1"]], True)[0], c["a1"]))
    back(0, g_a1, [c["in"]], False)
    grads = unet_flatten([(gw, gb) for gw, gb in zip(gconv, gbias)], ghead)
    return loss, grads
