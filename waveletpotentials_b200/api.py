"""Host-side mirror of the reference's C++ entry points for the projection-and-recovery path.

Class and method names follow the reference (CuWHHDForward::Solve1D, CuWaveletPotentialRecover3D,
CuDivLocalProject3D::ProjectLocal_q_ccc, CuMultigridFrac3D::Solve / GetResdualError,
CuConvergence::GetB_3d_frac_vel, CuGradient::Gradient3D_Frac_P, CuSolidLevelSet3D) so code written
against the reference reads the same.  Arguments are torch CUDA float32 tensors in the reference
layout: a 3D array with extents (DX, DY, DZ) has torch shape (DZ, DX, DY) (y contiguous); 2D arrays
are (DX, DY).  Every call goes through the C ABI of libwp_b200.so (include/wp_api.h); errors
raise WPError instead of exiting the process.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from ._lib import START_FMG, START_ZERO  # noqa: F401
from ._lib import WAIT_SITE_BATCH_PUBLISH, WAIT_SITE_CONV_PIPELINE, WAIT_SITE_GRID_BARRIER  # noqa: F401
from ._lib import BATCH_AUTO, BATCH_GRAPH, BATCH_PERSISTENT  # noqa: F401
from ._lib import CDF3_7, CDF4_6, PREC_FP32, PREC_FP64, PREC_MIXED, PROLONG_CONSTANT, PROLONG_TRILINEAR, MgParams, \
    MgReport, WPError, check, lib

__all__ = ["CuWHHDForward", "CuWaveletPotentialRecover3D", "CuWaveletPotentialRecover2D", "CuMultigridFrac3D",
           "CuMultigridFrac2D", "CuConvergence", "CuGradient", "CuSolidLevelSet3D", "CuSolidLevelSet2D", "CuDst3D",
           "Projector3D", "Projector2D", "BatchProjector", "max_abs", "conv3_forward", "conv3_wgrad",
           "random_field3d", "velocity3d_device", "UNetWarmStart", "warm_started_solve",
           "ip_diag", "WPError", "CDF3_7", "CDF4_6", "PREC_FP32", "PREC_MIXED", "PREC_FP64", "PROLONG_CONSTANT",
           "PROLONG_TRILINEAR", "START_ZERO", "START_FMG", "mac_shapes3d", "mac_shapes2d", "BATCH_GRAPH",
           "BATCH_PERSISTENT", "BATCH_AUTO"]


def mac_shapes3d(nx, ny, nz):
    return {"xv": (nz, nx + 1, ny), "yv": (nz, nx, ny + 1), "zv": (nz + 1, nx, ny),
            "qx": (nz + 1, nx, ny + 1), "qy": (nz + 1, nx + 1, ny), "qz": (nz, nx + 1, ny + 1), "p": (nz, nx, ny)}


def mac_shapes2d(nx, ny):
    return {"xv": (nx + 1, ny), "yv": (nx, ny + 1), "qz": (nx + 1, ny + 1), "p": (nx, ny)}


def _stream(stream):
    if stream is None:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _ptr(t: torch.Tensor | None, shape=None, dtype=torch.float32, name="tensor"):
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise WPError(1, name, "expected a CUDA tensor")
    if t.dtype != dtype:
        raise WPError(1, name, f"expected {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise WPError(1, name, "expected a contiguous tensor")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise WPError(1, name, f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
    return ctypes.c_void_p(t.data_ptr())


def _c(ch: str):
    return ctypes.c_char(ch.encode())


def _dims3(dim):
    nx, ny, nz = (int(v) for v in dim)
    return nx, ny, nz


def _dx3(dx):
    if isinstance(dx, (int, float)):
        return float(dx), float(dx), float(dx)
    return tuple(float(v) for v in dx)


class CuWHHDForward:
    """CuWHHDForward::Solve1D (cuWHHDForward.cu:1122-1153): full-depth 1D transform along one axis."""

    @staticmethod
    def Solve1D(dst, src, dim, level, direction, bc="n", rsw_type=CDF3_7, is_forward=True, stream=None):
        dx, dy, dz = _dims3(dim)
        src = dst if src is None else src
        dt = dst.dtype
        if dt not in (torch.float32, torch.float64):
            raise WPError(1, "Solve1D", "float32 or float64 tensors only")
        shape = (dz, dx, dy)
        fn = lib().wp_dwt1d if dt == torch.float32 else lib().wp_dwt1d_f64
        check(fn(_ptr(dst, shape, dt, "dst"), _ptr(src, shape, dt, "src"), dx, dy, dz, int(level),
                 _c(direction), _c(bc), int(rsw_type), int(bool(is_forward)), _stream(stream)), "wp_dwt1d")


def ip_diag(dim: int, wavelet: int, bc: str):
    """Diagonal inner-product table (CuGetInnerProduct::GenerateIp band 0), computed on the GPU."""
    import numpy as np
    out = np.zeros(int(dim))
    check(lib().wp_ip_diag(out.ctypes.data_as(ctypes.c_void_p), int(dim), int(wavelet), _c(bc)), "wp_ip_diag")
    return out


class CuWaveletPotentialRecover3D:
    """CuWaveletPotentialRecover3D (cuWaveletPotentialRecover3D.cuh:11-15)."""

    def __init__(self, dim, dx, bc="n", type_w_curl=CDF3_7, type_w_div=CDF4_6):
        self.dim = _dims3(dim)
        self.dx = _dx3(dx)
        self.shapes = mac_shapes3d(*self.dim)
        h = ctypes.c_void_p()
        check(lib().wp_recover3d_create(ctypes.byref(h), *self.dim, *self.dx, _c(bc), int(type_w_curl),
                                        int(type_w_div)), "wp_recover3d_create")
        self._h = h

    def Solve(self, qx, qy, qz, xv, yv, zv, stream=None):
        s = self.shapes
        check(lib().wp_recover3d_run(self._h, _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]),
                                     _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]), _stream(stream)),
              "wp_recover3d_run")

    def CutCoefficients(self, qx_out, qy_out, qz_out, qx, qy, qz, level, stream=None):
        """Coarse-scale part of a potential (cuWaveletPotentialRecover3D.cu:199-239): the wavelet
        coefficients below `level` cleared, synthesised back into the _out arrays."""
        s = self.shapes
        check(lib().wp_recover3d_cut(self._h, _ptr(qx_out, s["qx"]), _ptr(qy_out, s["qy"]), _ptr(qz_out, s["qz"]),
                                     _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]), int(level),
                                     _stream(stream)), "wp_recover3d_cut")

    def ProjectLocal_q_ccc(self, qx, qy, qz, xv_lwt, yv_lwt, zv_lwt, stream=None):
        s = self.shapes
        check(lib().wp_recover3d_project(self._h, _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]),
                                         _ptr(xv_lwt, s["xv"]), _ptr(yv_lwt, s["yv"]), _ptr(zv_lwt, s["zv"]),
                                         _stream(stream)), "wp_recover3d_project")

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_recover3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuWaveletPotentialRecover2D:
    """CuWaveletPotentialRecover2D (cuWaveletPotentialRecover2D.cuh:11-15)."""

    def __init__(self, dim, dx, bc="n", type_w_curl=CDF3_7, type_w_div=CDF4_6):
        self.dim = tuple(int(v) for v in dim)
        self.dx = (float(dx), float(dx)) if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
        self.shapes = mac_shapes2d(*self.dim)
        h = ctypes.c_void_p()
        check(lib().wp_recover2d_create(ctypes.byref(h), *self.dim, *self.dx, _c(bc), int(type_w_curl),
                                        int(type_w_div)), "wp_recover2d_create")
        self._h = h

    def Solve(self, qz, xv, yv, stream=None):
        s = self.shapes
        check(lib().wp_recover2d_run(self._h, _ptr(qz, s["qz"]), _ptr(xv, s["xv"]), _ptr(yv, s["yv"]),
                                     _stream(stream)), "wp_recover2d_run")

    def ProjectSingle(self, qz, xv_lwt, yv_lwt, stream=None):
        s = self.shapes
        check(lib().wp_recover2d_project(self._h, _ptr(qz, s["qz"]), _ptr(xv_lwt, s["xv"]), _ptr(yv_lwt, s["yv"]),
                                         _stream(stream)), "wp_recover2d_project")

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_recover2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _report(r: MgReport) -> dict:
    return {"cycles": r.cycles, "rel_residual": r.rel_residual, "history": list(r.history[:min(r.steps, 64)])}


class CuMultigridFrac3D:
    """CuMultigridFrac3D (cuMultigridFrac3D.cuh:15-18)."""

    def __init__(self, ax, ay, az, dim, dx, bc="n", stream=None):
        self.dim = _dims3(dim)
        self.dx = _dx3(dx)
        s = mac_shapes3d(*self.dim)
        self.cells = s["p"]
        h = ctypes.c_void_p()
        check(lib().wp_mgfrac3d_create(ctypes.byref(h), _ptr(ax, s["xv"], name="ax"), _ptr(ay, s["yv"], name="ay"),
                                       _ptr(az, s["zv"], name="az"), *self.dim, *self.dx, _c(bc), _stream(stream)),
              "wp_mgfrac3d_create")
        self._h = h

    def Solve(self, dst, pre_v, f, n_iters=10, nu1=2, nu2=2, weight=0.8, stream=None):
        """Exactly n_iters FP32 V-cycles of the reference algorithm (cuMultigridFrac3D.cu:249-265)."""
        c = self.cells
        check(lib().wp_mgfrac3d_solve(self._h, _ptr(dst, c), _ptr(pre_v, c), _ptr(f, c), int(n_iters), int(nu1),
                                      int(nu2), float(weight), _stream(stream)), "wp_mgfrac3d_solve")

    def Solve_index(self, dst, pre_v, f, n_iters=10, nu1=2, nu2=2, weight=0.8, stream=None):
        """n_iters index-sparse V-cycles over the cells with a face fraction >= 1e-12
        (CuMultigridFrac3D::Solve_index, cuMultigridFrac3D.cu:347-420): post-smoothing runs nu1
        sweeps as in the reference, unlisted cells keep their start value.  FP64 when dst is float64
        (the reference's default precision; pre_v and f then float64 too), else FP32."""
        c = self.cells
        fn = lib().wp_mgfrac3d_solve_index64 if dst.dtype == torch.float64 else lib().wp_mgfrac3d_solve_index
        dt = torch.float64 if dst.dtype == torch.float64 else torch.float32
        check(fn(self._h, _ptr(dst, c, dt), _ptr(pre_v, c, dt), _ptr(f, c, dt), int(n_iters), int(nu1), int(nu2),
                 float(weight), _stream(stream)), "wp_mgfrac3d_solve_index")

    def IndexSizes(self, stream=None):
        """(listed cells per level, listed 32-cell row segments per level) of the index-sparse cycle."""
        cells = (ctypes.c_longlong * 32)()
        segs = (ctypes.c_longlong * 32)()
        nl = ctypes.c_int()
        check(lib().wp_mgfrac3d_index_sizes(self._h, ctypes.cast(cells, ctypes.c_void_p),
                                            ctypes.cast(segs, ctypes.c_void_p), 32, ctypes.byref(nl),
                                            _stream(stream)), "wp_mgfrac3d_index_sizes")
        return [cells[k] for k in range(nl.value)], [segs[k] for k in range(nl.value)]

    def SolveTol(self, dst, pre_v, f, rel_tol=1e-6, max_cycles=50, nu1=2, nu2=2, weight=2.0 / 3.0,
                 precision=PREC_MIXED, prolongation=PROLONG_TRILINEAR, raise_on_fail=True, start=START_ZERO,
                 host_loop=False, inner_cycles=1, stream=None) -> dict:
        c = self.cells
        prm = MgParams(int(max_cycles), int(nu1), int(nu2), float(weight), float(rel_tol), int(precision),
                       int(prolongation), int(start), int(bool(host_loop)), int(inner_cycles))
        rep = MgReport()
        st = lib().wp_mgfrac3d_solve_tol(self._h, _ptr(dst, c), _ptr(pre_v, c), _ptr(f, c), ctypes.byref(prm),
                                         ctypes.byref(rep), _stream(stream))
        out = _report(rep)
        out["status"] = _lib.STATUS.get(st, st)
        if raise_on_fail and st != 0:
            check(st, "wp_mgfrac3d_solve_tol")
        return out

    def UniformRows(self, level=0):
        """(rows of the level whose face fractions are all 1, rows in all): the rows the column
        kernels stream without reading fractions."""
        u, r = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().wp_mgfrac3d_uniform_rows(self._h, int(level), ctypes.byref(u), ctypes.byref(r)),
              "wp_mgfrac3d_uniform_rows")
        return u.value, r.value

    def Autotune(self, stream=None):
        """Times the level kernels over candidate z-chunks and keeps the fastest (synchronous)."""
        check(lib().wp_mgfrac3d_autotune(self._h, _stream(stream)), "wp_mgfrac3d_autotune")

    def Tiles(self, with_times=False):
        """Per level: (jacobi, restrict, defect) z-chunks in use; with_times adds the kernel variants
        and the tuned times per sweep in ms."""
        buf = (ctypes.c_int * (3 * 32))()
        var = (ctypes.c_int * (3 * 32))()
        ms = (ctypes.c_float * (3 * 32))()
        nl = ctypes.c_int()
        check(lib().wp_mgfrac3d_tiles(self._h, ctypes.cast(buf, ctypes.c_void_p), ctypes.cast(var, ctypes.c_void_p),
                                      ctypes.cast(ms, ctypes.c_void_p), 96, ctypes.byref(nl)), "wp_mgfrac3d_tiles")
        zc = [tuple(buf[3 * l:3 * l + 3]) for l in range(nl.value)]
        if with_times:
            return (zc, [tuple(var[3 * l:3 * l + 3]) for l in range(nl.value)],
                    [tuple(round(v, 4) for v in ms[3 * l:3 * l + 3]) for l in range(nl.value)])
        return zc

    def SetTile(self, level, kind, zc, variant=0):
        """Pins one level's z-chunk and kernel variant (see wp_mgfrac3d_set_tile)."""
        check(lib().wp_mgfrac3d_set_tile(self._h, int(level), int(kind), int(zc), int(variant)),
              "wp_mgfrac3d_set_tile")

    def Iterate64Ptr(self) -> int:
        """Device address of the FP64 iterate of the last mixed / FP64 solve (no copy)."""
        out = ctypes.c_void_p()
        check(lib().wp_mgfrac3d_iterate64_view(self._h, ctypes.byref(out)), "wp_mgfrac3d_iterate64_view")
        return int(out.value)

    def Iterate64(self, stream=None):
        """FP64 iterate of the last mixed / FP64 solve, as a numpy array."""
        t = torch.empty(self.cells, device="cuda", dtype=torch.float64)
        check(lib().wp_mgfrac3d_iterate64(self._h, ctypes.c_void_p(t.data_ptr()), _stream(stream)),
              "wp_mgfrac3d_iterate64")
        return t.cpu().numpy()

    def GetResdualError(self, dst, f, stream=None) -> float:
        out = ctypes.c_double()
        c = self.cells
        check(lib().wp_mgfrac3d_residual(self._h, _ptr(dst, c), _ptr(f, c), ctypes.byref(out), _stream(stream)),
              "wp_mgfrac3d_residual")
        return out.value

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_mgfrac3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuMultigridFrac2D:
    """CuMultigridFrac2D (cuMultigridFrac2D.cuh:15-17)."""

    def __init__(self, ax, ay, dim, dx, bc="n", stream=None):
        self.dim = tuple(int(v) for v in dim)
        self.dx = (float(dx), float(dx)) if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
        s = mac_shapes2d(*self.dim)
        self.cells = s["p"]
        h = ctypes.c_void_p()
        check(lib().wp_mgfrac2d_create(ctypes.byref(h), _ptr(ax, s["xv"], name="ax"), _ptr(ay, s["yv"], name="ay"),
                                       *self.dim, *self.dx, _c(bc), _stream(stream)), "wp_mgfrac2d_create")
        self._h = h

    def Solve(self, dst, pre_v, f, n_iters=10, nu1=2, nu2=2, weight=0.8, stream=None):
        c = self.cells
        check(lib().wp_mgfrac2d_solve(self._h, _ptr(dst, c), _ptr(pre_v, c), _ptr(f, c), int(n_iters), int(nu1),
                                      int(nu2), float(weight), _stream(stream)), "wp_mgfrac2d_solve")

    def SolveTol(self, dst, pre_v, f, rel_tol=1e-6, max_cycles=50, nu1=2, nu2=2, weight=2.0 / 3.0,
                 precision=PREC_MIXED, prolongation=PROLONG_TRILINEAR, raise_on_fail=True, start=START_ZERO,
                 host_loop=False, inner_cycles=1, stream=None) -> dict:
        c = self.cells
        prm = MgParams(int(max_cycles), int(nu1), int(nu2), float(weight), float(rel_tol), int(precision),
                       int(prolongation), int(start), int(bool(host_loop)), int(inner_cycles))
        rep = MgReport()
        st = lib().wp_mgfrac2d_solve_tol(self._h, _ptr(dst, c), _ptr(pre_v, c), _ptr(f, c), ctypes.byref(prm),
                                         ctypes.byref(rep), _stream(stream))
        out = _report(rep)
        out["status"] = _lib.STATUS.get(st, st)
        if raise_on_fail and st != 0:
            check(st, "wp_mgfrac2d_solve_tol")
        return out

    def GetResdualError(self, dst, f, stream=None) -> float:
        out = ctypes.c_double()
        c = self.cells
        check(lib().wp_mgfrac2d_residual(self._h, _ptr(dst, c), _ptr(f, c), ctypes.byref(out), _stream(stream)),
              "wp_mgfrac2d_residual")
        return out.value

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_mgfrac2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuConvergence:
    """CuConvergence::GetB_3d_frac_vel / GetB_2d_frac_vel: b = -div(a u)."""

    @staticmethod
    def GetB_3d_frac_vel(b, xv, yv, zv, ax, ay, az, dim, dx, bc="n", stream=None):
        nx, ny, nz = _dims3(dim)
        s = mac_shapes3d(nx, ny, nz)
        check(lib().wp_divergence_frac3d(_ptr(b, s["p"]), _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]),
                                         _ptr(ax, s["xv"]), _ptr(ay, s["yv"]), _ptr(az, s["zv"]), nx, ny, nz,
                                         *_dx3(dx), _stream(stream)), "wp_divergence_frac3d")

    @staticmethod
    def GetB_2d_frac_vel(b, xv, yv, ax, ay, dim, dx, bc="n", stream=None):
        nx, ny = (int(v) for v in dim)
        s = mac_shapes2d(nx, ny)
        d = (float(dx), float(dx)) if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
        check(lib().wp_divergence_frac2d(_ptr(b, s["p"]), _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(ax, s["xv"]),
                                         _ptr(ay, s["yv"]), nx, ny, *d, _stream(stream)), "wp_divergence_frac2d")


class CuGradient:
    """CuGradient::Gradient3D_Frac_P + CudaMatAdd(-1) + CudaMatMul(a), fused: u <- (u - grad p) [* a]."""

    @staticmethod
    def SubtractGradient3D_Frac_P(xv, yv, zv, p, ax, ay, az, dim, dx, multiply_frac=True, stream=None):
        nx, ny, nz = _dims3(dim)
        s = mac_shapes3d(nx, ny, nz)
        check(lib().wp_grad_subtract_frac3d(_ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]), _ptr(p, s["p"]),
                                            _ptr(ax, s["xv"]), _ptr(ay, s["yv"]), _ptr(az, s["zv"]), nx, ny, nz,
                                            *_dx3(dx), int(bool(multiply_frac)), _stream(stream)),
              "wp_grad_subtract_frac3d")

    @staticmethod
    def SubtractGradient3D_Frac_P64(xv, yv, zv, p64_ptr, ax, ay, az, dim, dx, multiply_frac=True, stream=None):
        """The same update with an FP64 pressure given by its device address (the solver's FP64
        iterate, CuMultigridFrac3D.Iterate64Ptr): formed in FP64, rounded once per face."""
        nx, ny, nz = _dims3(dim)
        s = mac_shapes3d(nx, ny, nz)
        check(lib().wp_grad_subtract_frac3d_p64(_ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]),
                                                ctypes.c_void_p(int(p64_ptr)), _ptr(ax, s["xv"]), _ptr(ay, s["yv"]),
                                                _ptr(az, s["zv"]), nx, ny, nz, *_dx3(dx), int(bool(multiply_frac)),
                                                _stream(stream)),
              "wp_grad_subtract_frac3d_p64")

    @staticmethod
    def SubtractGradient2D_Frac_P(xv, yv, p, ax, ay, dim, dx, multiply_frac=True, stream=None):
        nx, ny = (int(v) for v in dim)
        s = mac_shapes2d(nx, ny)
        d = (float(dx), float(dx)) if isinstance(dx, (int, float)) else tuple(float(v) for v in dx)
        check(lib().wp_grad_subtract_frac2d(_ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(p, s["p"]), _ptr(ax, s["xv"]),
                                            _ptr(ay, s["yv"]), nx, ny, *d, int(bool(multiply_frac)),
                                            _stream(stream)), "wp_grad_subtract_frac2d")


def max_abs(t: torch.Tensor, stream=None) -> float:
    """CudaFindMaxValue without the host copy of the array."""
    out = ctypes.c_double()
    check(lib().wp_max_abs(_ptr(t), t.numel(), ctypes.byref(out), _stream(stream)), "wp_max_abs")
    return out.value


class CuSolidLevelSet3D:
    """CuSolidLevelSet3D: sphere level set (positive in fluid) and face open fractions."""

    def __init__(self, dim, dx):
        self.dim = _dims3(dim)
        self.dx = float(dx)
        nx, ny, nz = self.dim
        self.ls = torch.empty((nz, nx, ny), device="cuda", dtype=torch.float32)

    def InitLsSpheres(self, centers, radii, stream=None):
        import numpy as np
        c = np.ascontiguousarray(np.reshape(centers, (-1, 3)), dtype=np.float64)
        r = np.ascontiguousarray(np.reshape(radii, (-1,)), dtype=np.float64)
        check(lib().wp_sdf_spheres3d(_ptr(self.ls), *self.dim, self.dx, c.ctypes.data_as(ctypes.c_void_p),
                                     r.ctypes.data_as(ctypes.c_void_p), int(r.size), _stream(stream)),
              "wp_sdf_spheres3d")

    def InitLsSphere(self, center, radius, stream=None):
        self.InitLsSpheres([center], [radius], stream)

    def GetFrac(self, ax, ay, az, ls=None, dim=None, dx=None, stream=None):
        """GetFrac(ax, ay, az): fractions of the object's level set from the values at the two cells
        of each face (cuGetAx/Ay/Az).  GetFrac(ax, ay, az, ls, dim, dx): the reference's static
        overload for an arbitrary level set, sub-sampling the cut faces (cuGetAx/Ay/Az_divide)."""
        if ls is None:
            s = mac_shapes3d(*self.dim)
            check(lib().wp_fractions3d(_ptr(ax, s["xv"]), _ptr(ay, s["yv"]), _ptr(az, s["zv"]), _ptr(self.ls),
                                       *self.dim, self.dx, _stream(stream)), "wp_fractions3d")
            return
        d = _dims3(dim) if dim is not None else self.dim
        h = float(dx) if dx is not None else self.dx
        s = mac_shapes3d(*d)
        check(lib().wp_fractions3d_subsampled(_ptr(ax, s["xv"]), _ptr(ay, s["yv"]), _ptr(az, s["zv"]),
                                              _ptr(ls, s["p"]), *d, h, _stream(stream)), "wp_fractions3d_subsampled")


    def AddBoxes(self, lo, hi, stream=None):
        """Union of axis-aligned boxes into the level set (no reference counterpart)."""
        import numpy as np
        l = np.ascontiguousarray(np.reshape(lo, (-1, 3)), dtype=np.float64)
        u = np.ascontiguousarray(np.reshape(hi, (-1, 3)), dtype=np.float64)
        check(lib().wp_sdf_boxes3d(_ptr(self.ls), *self.dim, self.dx, l.ctypes.data_as(ctypes.c_void_p),
                                   u.ctypes.data_as(ctypes.c_void_p), int(l.shape[0]), _stream(stream)),
              "wp_sdf_boxes3d")


class CuFastSweeping:
    """CuFastSweeping (cuFastSweeping.cu): eikonal redistancing of a level set (torch CUDA float32,
    shape (DZ, DX, DY)) in place."""

    @staticmethod
    def Solve(ls, dim, dx, n_iters, stream=None):
        d = _dims3(dim)
        check(lib().wp_fast_sweep_solve(_ptr(ls, (d[2], d[0], d[1])), *d, float(dx), int(n_iters), _stream(stream)),
              "wp_fast_sweep_solve")

    @staticmethod
    def ReinitLevelSet(ls, dim, dx, n_iters, stream=None):
        d = _dims3(dim)
        check(lib().wp_fast_sweep_reinit(_ptr(ls, (d[2], d[0], d[1])), *d, float(dx), int(n_iters),
                                         _stream(stream)), "wp_fast_sweep_reinit")


def ParticlesToLs(ls, x, dim, dx, radius, max_dis, n_iters, stream=None):
    """CuFastSweeping::ParticlesToLs: ls (CUDA float32 (DZ, DX, DY)) from particle positions x (CUDA
    float32 (count, 3))."""
    d = _dims3(dim)
    count = int(x.shape[0])
    check(lib().wp_particles_to_ls(_ptr(ls, (d[2], d[0], d[1])), _ptr(x, (count, 3)), count, *d, float(dx),
                                   float(radius), float(max_dis), int(n_iters), _stream(stream)),
          "wp_particles_to_ls")


CuFastSweeping.ParticlesToLs = staticmethod(ParticlesToLs)


def ParticlesToLsNarrow(ls, x, dim, dx, radius, max_dis, n_iters, stream=None):
    """CuFastSweeping::ParticlesToLsNarrow: ls (CUDA float32 (DZ, DX, DY)) holds the start and receives
    the level set of the particles x (CUDA float32 (count, 3))."""
    d = _dims3(dim)
    count = int(x.shape[0])
    check(lib().wp_particles_to_ls_narrow(_ptr(ls, (d[2], d[0], d[1])), _ptr(x, (count, 3)), count, *d, float(dx),
                                          float(radius), float(max_dis), int(n_iters), _stream(stream)),
          "wp_particles_to_ls_narrow")


CuFastSweeping.ParticlesToLsNarrow = staticmethod(ParticlesToLsNarrow)


class CuSolidLevelSet2D:
    """CuSolidLevelSet2D: circle level set (positive in fluid) and face open fractions."""

    def __init__(self, dim, dx):
        self.dim = tuple(int(v) for v in dim)
        self.dx = float(dx)
        self.ls = torch.empty(self.dim, device="cuda", dtype=torch.float32)

    def InitLsCircles(self, centers, radii, stream=None):
        import numpy as np
        c = np.ascontiguousarray(np.reshape(centers, (-1, 2)), dtype=np.float64)
        r = np.ascontiguousarray(np.reshape(radii, (-1,)), dtype=np.float64)
        check(lib().wp_sdf_circles2d(_ptr(self.ls), *self.dim, self.dx, c.ctypes.data_as(ctypes.c_void_p),
                                     r.ctypes.data_as(ctypes.c_void_p), int(r.size), _stream(stream)),
              "wp_sdf_circles2d")

    def GetFrac(self, ax, ay, stream=None):
        s = mac_shapes2d(*self.dim)
        check(lib().wp_fractions2d(_ptr(ax, s["xv"]), _ptr(ay, s["yv"]), _ptr(self.ls), *self.dim, self.dx,
                                   _stream(stream)), "wp_fractions2d")


class CuDst3D:
    """CuDst3D (cuDst3D.cuh): Dirichlet Poisson solve by DST-I, FP64 tensors of shape (nz, nx, ny)."""

    def __init__(self, dim, dx):
        self.dim = _dims3(dim)
        self.dx = _dx3(dx)
        h = ctypes.c_void_p()
        check(lib().wp_dst3d_create(ctypes.byref(h), *self.dim, *self.dx), "wp_dst3d_create")
        self._h = h

    def Solve(self, dst, f, stream=None):
        nx, ny, nz = self.dim
        check(lib().wp_dst3d_solve(self._h, _ptr(dst, (nz, nx, ny), torch.float64), _ptr(f, (nz, nx, ny), torch.float64),
                                   _stream(stream)), "wp_dst3d_solve")

    @staticmethod
    def SolveNoAlloc(dst, f, dim, dx, stream=None):
        """Handle-free solve with no device allocation (grids up to 64 per axis, 64^3 cells)."""
        nx, ny, nz = _dims3(dim)
        check(lib().wp_dst3d_solve_noalloc(_ptr(dst, (nz, nx, ny), torch.float64),
                                           _ptr(f, (nz, nx, ny), torch.float64), nx, ny, nz, *_dx3(dx),
                                           _stream(stream)), "wp_dst3d_solve_noalloc")

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_dst3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuParallelSweep3D:
    """CuParallelSweep3D (cuParallelSweep3D.cuh): the sweep + DST-I potential recovery, the
    reference's comparison baseline for the wavelet recovery (bc 'n').  3D: Solve then Project gives
    a divergence-free vector potential with curl q = u; 2D: Solve2D (qz from the velocity)."""

    def __init__(self, dim, dx, bc="n"):
        self.dim = _dims3(dim)
        self.dx = _dx3(dx)
        h = ctypes.c_void_p()
        check(lib().wp_sweep3d_create(ctypes.byref(h), *self.dim, *self.dx, _c(bc)), "wp_sweep3d_create")
        self._h = h
        self.shapes = mac_shapes3d(*self.dim)

    def Solve(self, qx, qy, qz, xv, yv, zv, stream=None):
        s = self.shapes
        check(lib().wp_sweep3d_solve(self._h, _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]),
                                     _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]), _stream(stream)),
              "wp_sweep3d_solve")

    def SolveFromMid(self, qx, qy, qz, xv, yv, zv, mid, stream=None):
        """CuParallelSweep3D::SolveFromMid: the integrals run both ways from plane mid[2] (and row
        mid[0] of qy's plane there); mid[1] is unused."""
        s = self.shapes
        mx, my, mz = (int(v) for v in mid)
        check(lib().wp_sweep3d_solve_from_mid(self._h, _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]),
                                              _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]), mx, my, mz,
                                              _stream(stream)), "wp_sweep3d_solve_from_mid")

    def Project(self, qx, qy, qz, stream=None):
        s = self.shapes
        check(lib().wp_sweep3d_project(self._h, _ptr(qx, s["qx"]), _ptr(qy, s["qy"]), _ptr(qz, s["qz"]),
                                       _stream(stream)), "wp_sweep3d_project")

    @staticmethod
    def Solve2D(qz, xv, yv, dim, dx, bc="n", stream=None):
        nx, ny = (int(v) for v in dim)
        d = (float(dx), float(dx)) if not isinstance(dx, (tuple, list)) else (float(dx[0]), float(dx[1]))
        s = mac_shapes2d(nx, ny)
        check(lib().wp_sweep2d_solve(_ptr(qz, s["qz"]), _ptr(xv, s["xv"]), _ptr(yv, s["yv"]), nx, ny, *d, _c(bc),
                                     _stream(stream)), "wp_sweep2d_solve")

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_sweep3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


WARM_START_ACCEPT = 0.3  # relative residual after one V-cycle below which the network's guess is kept


def warm_started_solve(mg, p, b, sdf, hcell, net, opts, stream=None) -> dict:
    """Multigrid solve to the same tolerance from the network's guess, with the plain solver as
    fallback: one V-cycle from the guess (its first pre-smoothing removes the guess's grid-scale
    noise); if the residual is then not below WARM_START_ACCEPT (about one V-cycle's reduction from a
    zero start) the solve restarts from zero, otherwise it continues from that iterate."""
    net.predict(p, b, sdf, hcell, stream)
    one = dict(opts)
    one["max_cycles"] = 1
    one["rel_tol"] = 0.0
    first = mg.SolveTol(p, p, b, raise_on_fail=False, stream=stream, **one)
    r1 = first["rel_residual"]
    used = bool(r1 < WARM_START_ACCEPT)
    if used:
        rest = dict(opts)
        rest["max_cycles"] = max(1, opts.get("max_cycles", 60) - 1)
        rep = mg.SolveTol(p, p, b, raise_on_fail=False, stream=stream, **rest)
        rep["cycles"] += 1
        rep["history"] = first["history"] + rep["history"]
    else:
        rep = mg.SolveTol(p, None, b, raise_on_fail=False, stream=stream, **opts)
        rep["cycles"] += 1  # the discarded cycle from the guess
    rep["warm_start"] = {"first_cycle_rel_residual": r1, "used": used}
    return rep


class Projector3D:
    """One projection of a MAC velocity field (the composition of TestLocalProjection.cpp:666-767):
    b = -div(a u) -> fractional multigrid solve to tolerance -> u <- a (u - grad p) -> max|div| check
    -> wavelet potential recovery q.
    """

    def __init__(self, ax, ay, az, dim, dx, rel_tol=1e-6, max_cycles=60, nu1=2, nu2=2, weight=2.0 / 3.0,
                 precision=PREC_MIXED, prolongation=PROLONG_TRILINEAR, autotune=True, warm_start=None, sdf=None,
                 start=START_ZERO, host_loop=False, inner_cycles=1,
                 stream=None):
        self.dim = _dims3(dim)
        self.dx = _dx3(dx)
        self.ax, self.ay, self.az = ax, ay, az
        if warm_start is not None and sdf is None:
            raise WPError(1, "Projector3D", "a warm start needs the solid level set (sdf)")
        self.warm_start, self.sdf = warm_start, sdf
        self.mg = CuMultigridFrac3D(ax, ay, az, self.dim, self.dx, "n", stream)
        if autotune:
            self.mg.Autotune(stream)
        self.rec = CuWaveletPotentialRecover3D(self.dim, self.dx, "n")
        self.opts = dict(rel_tol=rel_tol, max_cycles=max_cycles, nu1=nu1, nu2=nu2, weight=weight, precision=precision,
                         prolongation=prolongation, start=start, host_loop=host_loop, inner_cycles=inner_cycles)
        s = mac_shapes3d(*self.dim)
        self.shapes = s
        self.b = torch.empty(s["p"], device="cuda", dtype=torch.float32)
        self.p = torch.empty(s["p"], device="cuda", dtype=torch.float32)

    def run(self, xv, yv, zv, qx, qy, qz, pre_p=None, stream=None) -> dict:
        """Projects (xv, yv, zv) in place (result a (u - grad p)) and writes the potential q."""
        CuConvergence.GetB_3d_frac_vel(self.b, xv, yv, zv, self.ax, self.ay, self.az, self.dim, self.dx,
                                       stream=stream)
        if pre_p is None and self.warm_start is not None:
            rep = warm_started_solve(self.mg, self.p, self.b, self.sdf, self.dx[0], self.warm_start, self.opts,
                                     stream)
        else:
            rep = self.mg.SolveTol(self.p, pre_p, self.b, raise_on_fail=False, stream=stream, **self.opts)
        if self.opts["precision"] != PREC_FP32:
            # the gradient of the FP64 iterate, formed in FP64 (the FP32 copy's rounding, amplified by
            # the 1/h of the difference, would dominate the projected field's divergence)
            CuGradient.SubtractGradient3D_Frac_P64(xv, yv, zv, self.mg.Iterate64Ptr(), self.ax, self.ay, self.az,
                                                   self.dim, self.dx, multiply_frac=True, stream=stream)
        else:
            CuGradient.SubtractGradient3D_Frac_P(xv, yv, zv, self.p, self.ax, self.ay, self.az, self.dim, self.dx,
                                                 multiply_frac=True, stream=stream)
        # -div of the fraction-weighted projected field (open-face divergence of a (u - grad p))
        CuConvergence.GetB_3d_frac_vel(self.b, xv, yv, zv, None, None, None, self.dim, self.dx, stream=stream)
        rep["max_abs_div"] = max_abs(self.b, stream)
        self.rec.Solve(qx, qy, qz, xv, yv, zv, stream)
        return rep


class HostPipeline3D:
    """Projections of host-resident velocity fields through one Projector3D, with the transfers
    overlapped: the pinned host-to-device copy of step k+1 runs on one copy stream and the
    device-to-host copy of step k-1's potential on another while step k projects on the compute
    stream (two device buffer sets; the copy engines and the SMs work at the same time).  Each step
    copies its whole input in and its whole potential out; results are those of Projector3D.run.
    """

    def __init__(self, projector: "Projector3D", stream=None):
        self.pr = projector
        s = projector.shapes
        self.u = [[torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")] for _ in range(2)]
        self.q = [[torch.empty(s[k], device="cuda") for k in ("qx", "qy", "qz")] for _ in range(2)]
        self.comp = stream if stream is not None else torch.cuda.Stream()
        self.s_in, self.s_out = torch.cuda.Stream(), torch.cuda.Stream()
        ev = lambda timing=False: [torch.cuda.Event(enable_timing=timing) for _ in range(2)]
        self.ev_in, self.ev_done, self.ev_out = ev(), ev(), ev(True)
        self.last_out = None  # event after the last potential copied out by run()
        self.h2d_bytes = sum(4 * math.prod(s[k]) for k in ("xv", "yv", "zv"))
        self.d2h_bytes = sum(4 * math.prod(s[k]) for k in ("qx", "qy", "qz"))

    def _copy_in(self, k, host_u):
        b = k % 2
        with torch.cuda.stream(self.s_in):
            # buffer b was last projected at step k-2 (the projection writes u in place)
            self.s_in.wait_event(self.ev_done[b])
            for d, h in zip(self.u[b], host_u):
                d.copy_(h, non_blocking=True)
            self.ev_in[b].record(self.s_in)

    def run(self, host_in, host_out) -> list:
        """host_in[k] = (xv, yv, zv), host_out[k] = (qx, qy, qz): pinned CPU float32 tensors of the
        MAC shapes (the same tensors may repeat).  Returns the per-step reports; host_out holds the
        potentials once the call returns."""
        n = len(host_in)
        if len(host_out) != n:
            raise WPError(1, "HostPipeline3D.run", "host_in and host_out differ in length")
        for e in self.ev_done + self.ev_out:
            e.record(self.comp)
        reps = []
        if n:
            self._copy_in(0, host_in[0])
        for k in range(n):
            b = k % 2
            if k + 1 < n:
                self._copy_in(k + 1, host_in[k + 1])
            self.comp.wait_event(self.ev_in[b])
            self.comp.wait_event(self.ev_out[b])  # q[b] was read out at step k-2
            reps.append(self.pr.run(*self.u[b], *self.q[b], stream=self.comp))
            self.ev_done[b].record(self.comp)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(self.ev_done[b])
                for h, d in zip(host_out[k], self.q[b]):
                    h.copy_(d, non_blocking=True)
                self.ev_out[b].record(self.s_out)
            self.last_out = self.ev_out[b]
        self.s_out.synchronize()
        return reps


class Projector2D:
    """2D form of Projector3D (CuMultigridFrac2D + CuWaveletPotentialRecover2D)."""

    def __init__(self, ax, ay, dim, dx, rel_tol=1e-6, max_cycles=60, nu1=2, nu2=2, weight=2.0 / 3.0,
                 precision=PREC_MIXED, prolongation=PROLONG_TRILINEAR, start=START_ZERO, host_loop=False, inner_cycles=1,
                 stream=None):
        self.dim = tuple(int(v) for v in dim)
        self.dx = float(dx)
        self.ax, self.ay = ax, ay
        self.mg = CuMultigridFrac2D(ax, ay, self.dim, self.dx, "n", stream)
        self.rec = CuWaveletPotentialRecover2D(self.dim, self.dx, "n")
        self.opts = dict(rel_tol=rel_tol, max_cycles=max_cycles, nu1=nu1, nu2=nu2, weight=weight, precision=precision,
                         prolongation=prolongation, start=start, host_loop=host_loop, inner_cycles=inner_cycles)
        s = mac_shapes2d(*self.dim)
        self.b = torch.empty(s["p"], device="cuda", dtype=torch.float32)
        self.p = torch.empty(s["p"], device="cuda", dtype=torch.float32)

    def run(self, xv, yv, qz, pre_p=None, stream=None) -> dict:
        CuConvergence.GetB_2d_frac_vel(self.b, xv, yv, self.ax, self.ay, self.dim, self.dx, stream=stream)
        rep = self.mg.SolveTol(self.p, pre_p, self.b, raise_on_fail=False, stream=stream, **self.opts)
        CuGradient.SubtractGradient2D_Frac_P(xv, yv, self.p, self.ax, self.ay, self.dim, self.dx, multiply_frac=True,
                                             stream=stream)
        CuConvergence.GetB_2d_frac_vel(self.b, xv, yv, None, None, self.dim, self.dx, stream=stream)
        rep["max_abs_div"] = max_abs(self.b, stream)
        self.rec.Solve(qz, xv, yv, stream)
        return rep


def _parray(ptrs):
    arr = (ctypes.c_void_p * len(ptrs))(*[p.value if isinstance(p, ctypes.c_void_p) else p for p in ptrs])
    return arr


class BatchProjector:
    """Many independent projections of uneven 2D/3D grids launched as one CUDA graph (wp_batch_*).

    ``grids`` is a list of dicts ``{"dim": (nx, ny[, nz]), "dx": h, "ax": ..., "ay": ...[, "az": ...]}``;
    a grid is 3D when its ``dim`` has three extents.  ``run(fields, outs)`` projects every grid in place
    and writes its potential, each grid's solve a device loop that stops at ``rel_tol`` (or
    ``max_cycles``) on the current input; ``plan(fields)`` (optional) measures the cycles of a
    representative input to order the grids over the graph's branches.  ``fields[i]`` is
    ``(xv, yv, zv)`` (3D) or ``(xv, yv)`` (2D); ``outs[i]`` is ``(qx, qy, qz)`` or ``(qz,)``.
    ``inner_cycles``: FP32 V-cycles per FP64 refinement step.  ``persistent``: every grid's solve in
    one persistent kernel inside the graph that takes (grid, level, pass) tiles from a device work
    queue (``wp_batch_set_mode(..., WP_BATCH_PERSISTENT, tile_cells)``), instead of a device loop of
    launches per grid; ``tile_cells`` (0 = the library's default) sets the cells per queue tile.
    ``mode`` ``BATCH_AUTO``: ``plan()`` times both ways on its inputs and the faster one runs.
    """

    def __init__(self, grids, rel_tol=1e-6, max_cycles=60, nu1=2, nu2=2, weight=2.0 / 3.0,
                 prolongation=PROLONG_TRILINEAR, nstreams=8, start=START_ZERO, inner_cycles=1,
                 persistent=False, tile_cells=0, mode=None):
        self.grids = grids
        self.count = len(grids)
        self.rel_tol = float(rel_tol)
        dims, ext, dx, ax, ay, az = [], [], [], [], [], []
        self.shapes = []
        for g in grids:
            d = tuple(int(v) for v in g["dim"])
            if len(d) == 3:
                s = mac_shapes3d(*d)
                dims.append(3)
                ext += list(d)
                az.append(_ptr(g["az"], s["zv"], name="az").value)
            else:
                s = mac_shapes2d(*d)
                dims.append(2)
                ext += [d[0], d[1], 1]
                az.append(None)
            self.shapes.append(s)
            dx.append(float(g["dx"]))
            ax.append(_ptr(g["ax"], s["xv"], name="ax").value)
            ay.append(_ptr(g["ay"], s["yv"], name="ay").value)
        self.dims = dims
        prm = MgParams(int(max_cycles), int(nu1), int(nu2), float(weight), float(rel_tol), PREC_MIXED,
                       int(prolongation), int(start), 0, int(inner_cycles))
        h = ctypes.c_void_p()
        self._keep = ((ctypes.c_int * self.count)(*dims), (ctypes.c_int * (3 * self.count))(*ext),
                      (ctypes.c_double * self.count)(*dx), _parray(ax), _parray(ay), _parray(az), prm)
        k = self._keep
        check(lib().wp_batch_create(ctypes.byref(h), self.count, ctypes.cast(k[0], ctypes.c_void_p),
                                    ctypes.cast(k[1], ctypes.c_void_p), ctypes.cast(k[2], ctypes.c_void_p),
                                    ctypes.cast(k[3], ctypes.c_void_p), ctypes.cast(k[4], ctypes.c_void_p),
                                    ctypes.cast(k[5], ctypes.c_void_p), ctypes.byref(prm), int(nstreams)),
              "wp_batch_create")
        self._h = h
        if persistent or mode is not None:
            self.set_mode(BATCH_PERSISTENT if persistent else mode, tile_cells)

    TILE_CANDIDATES = (4096, 8192, 16384, 32768, 65536)
    PROFILE_NAMES = ("init", "defect", "sweep0", "sweep", "sweep_acc", "restrict", "prolong", "coarse", "convert")

    def profile(self, enable, stream=None):
        """Persistent mode: the persistent kernel's activity counters since counting was last enabled
        (wp_batch_profile), as a dict of SM cycles summed over the CTAs; ``enable`` True clears them and
        counts the following runs, False stops."""
        out = (ctypes.c_double * 22)()
        check(lib().wp_batch_profile(self._h, 1 if enable else 0, ctypes.cast(out, ctypes.c_void_p), 22,
                                     _stream(stream)), "wp_batch_profile")
        v = list(out)
        d = {"wait_cycles": v[0], "tiles": v[1], "setup_cycles": v[2], "complete_cycles": v[3]}
        for k, nm in enumerate(self.PROFILE_NAMES):
            d[nm] = {"cycles": v[4 + 2 * k], "tiles": v[5 + 2 * k]}
        return d

    def get_mode(self):
        """(mode the batch runs in, cells per work-queue tile, the persistent tile timings in ms for
        ``TILE_CANDIDATES``, the graph mode's solve timing in ms) (wp_batch_get_mode); in persistent or
        auto mode with ``tile_cells`` 0, ``plan()`` times the candidate tiles and keeps the fastest, and
        in auto mode also the graph mode's solves, and runs the faster mode."""
        m = ctypes.c_int()
        t = ctypes.c_longlong()
        ms = (ctypes.c_float * 6)()
        check(lib().wp_batch_get_mode(self._h, ctypes.byref(m), ctypes.byref(t), ctypes.cast(ms, ctypes.c_void_p)),
              "wp_batch_get_mode")
        return m.value, t.value, list(ms)[:5], ms[5]

    def set_mode(self, mode, tile_cells=0):
        """BATCH_GRAPH or BATCH_PERSISTENT (see the class docstring); raises WPError (the mode
        unchanged) when a grid's levels do not fit the persistent program."""
        check(lib().wp_batch_set_mode(self._h, int(mode), int(tile_cells)), "wp_batch_set_mode")
        self.mode = int(mode)

    def _fields(self, fields, outs=None):
        names_in = ("xv", "yv", "zv")
        cols = [[], [], [], [], [], []]
        for i, s in enumerate(self.shapes):
            f = fields[i]
            d3 = self.dims[i] == 3
            for a in range(3):
                cols[a].append(_ptr(f[a], s[names_in[a]], name=names_in[a]).value if (a < 2 or d3) else None)
            if outs is not None:
                o = outs[i]
                if d3:
                    for a, nm in enumerate(("qx", "qy", "qz")):
                        cols[3 + a].append(_ptr(o[a], s[nm], name=nm).value)
                else:
                    cols[3].append(None)
                    cols[4].append(None)
                    cols[5].append(_ptr(o[0], s["qz"], name="qz").value)
        return [_parray(c) for c in cols]

    def plan(self, fields, stream=None):
        """Eager tolerance-driven pass on representative fields; returns each grid's V-cycles (fields
        unchanged).  Optional: the counts only order the grids over the graph's branches."""
        c = self._fields(fields)
        cyc = (ctypes.c_int * self.count)()
        check(lib().wp_batch_plan(self._h, ctypes.cast(c[0], ctypes.c_void_p), ctypes.cast(c[1], ctypes.c_void_p),
                                  ctypes.cast(c[2], ctypes.c_void_p), ctypes.cast(cyc, ctypes.c_void_p),
                                  _stream(stream)), "wp_batch_plan")
        return list(cyc)

    def run(self, fields, outs, stream=None):
        c = self._fields(fields, outs)
        self._last = c
        check(lib().wp_batch_run(self._h, *[ctypes.cast(a, ctypes.c_void_p) for a in c], _stream(stream)),
              "wp_batch_run")

    def results(self, stream=None) -> dict:
        """Per-grid max|div|, relative residual and V-cycles of the last run (each grid's device loop
        stops at ``rel_tol`` or ``max_cycles``).  ``over_tol[i]`` is true for a grid whose residual is
        still above ``rel_tol`` and ``status`` is then ``WP_ERR_NOT_CONVERGED``.  Any other failure
        raises."""
        m = (ctypes.c_double * self.count)()
        r = (ctypes.c_double * self.count)()
        cyc = (ctypes.c_int * self.count)()
        st = lib().wp_batch_results(self._h, ctypes.cast(m, ctypes.c_void_p), ctypes.cast(r, ctypes.c_void_p),
                                    ctypes.cast(cyc, ctypes.c_void_p), _stream(stream))
        if st != _lib.WP_ERR_NOT_CONVERGED:
            check(st, "wp_batch_results")
        rel = list(r)
        over = [self.rel_tol > 0 and not (x <= self.rel_tol) for x in rel]
        return {"max_abs_div": list(m), "rel_residual": rel, "cycles": list(cyc), "over_tol": over,
                "status": _lib.STATUS.get(st, st)}

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ test-only failure injection
def debug_withhold_wait(site, at=0, limit_s=1e-3):
    """Test only: the next launch at ``site`` (``WAIT_SITE_GRID_BARRIER``: the persistent
    below-finest multigrid cycle; ``WAIT_SITE_CONV_PIPELINE``: the tensor-core convolutions) leaves
    one wait without its arrival, so that wait runs out after ``limit_s`` and the call that launched
    it reports ``WP_ERR_DEVICE_WAIT``.  One shot; ``site`` 0 disarms (wp_debug_withhold_wait)."""
    check(lib().wp_debug_withhold_wait(int(site), int(at), float(limit_s)), "wp_debug_withhold_wait")


# ------------------------------------------------------------------ tensor-core convolutions
def _bf16(t, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.bfloat16 or not t.is_contiguous():
        raise WPError(1, name, "expected a contiguous CUDA bfloat16 tensor")
    return ctypes.c_void_p(t.data_ptr())


def conv3_forward(out, x0, w0, bias=None, x1=None, w1=None, relu=False, addend=None, mask=None, stream=None):
    """3x3x3 zero-padded convolution on the tensor cores.  x: (nz, nx, ny, cin) bf16 channels-last,
    w: (27, cout, cin) bf16, bias: (cout,) float32, out: (nz, nx, ny, cout) bf16."""
    nz, nx, ny, cin0 = x0.shape
    cout = w0.shape[1]
    cin1 = x1.shape[3] if x1 is not None else 0
    check(lib().wp_conv3_forward(_bf16(out, "out"), _bf16(x0, "x0"), cin0, _bf16(w0, "w0"),
                                 _bf16(x1, "x1") if x1 is not None else None, cin1,
                                 _bf16(w1, "w1") if w1 is not None else None,
                                 _ptr(bias, (cout,), name="bias") if bias is not None else None, cout, nx, ny, nz,
                                 int(bool(relu)), _bf16(addend, "addend") if addend is not None else None,
                                 _bf16(mask, "mask") if mask is not None else None, _stream(stream)),
          "wp_conv3_forward")


def conv3_wgrad(dw, x, gy, stream=None):
    """dw (27, cout, cin) float32 += weight gradient of the convolution for input x and output grad gy."""
    nz, nx, ny, cin = x.shape
    cout = gy.shape[3]
    check(lib().wp_conv3_wgrad(_ptr(dw, (27, cout, cin), name="dw"), _bf16(x, "x"), cin, _bf16(gy, "gy"), cout, nx, ny,
                               nz, _stream(stream)), "wp_conv3_wgrad")


# ------------------------------------------------------------------ seeded device generators
def random_field3d(out, slope, rms, kmax=8, seed=0, stream=None):
    """Gaussian random field (spectrum |k|^slope, |k| <= kmax, variance rms^2) into out (nz, nx, ny)."""
    nz, nx, ny = out.shape
    check(lib().wp_random_field3d(_ptr(out), nx, ny, nz, float(slope), float(rms), int(kmax), int(seed),
                                  _stream(stream)), "wp_random_field3d")


def velocity3d_device(xv, yv, zv, dim, seed, psi_slope=-11.0 / 3.0, psi_rms=1.0, phi_slope=-2.0, phi_rms=1.0, kmax=8,
                      stream=None):
    """MAC velocity u = curl(psi) + grad(phi) generated on the GPU (wp_velocity3d)."""
    nx, ny, nz = _dims3(dim)
    s = mac_shapes3d(nx, ny, nz)
    check(lib().wp_velocity3d(_ptr(xv, s["xv"]), _ptr(yv, s["yv"]), _ptr(zv, s["zv"]), nx, ny, nz, int(seed),
                              float(psi_slope), float(psi_rms), float(phi_slope), float(phi_rms), int(kmax),
                              _stream(stream)), "wp_velocity3d")


# ------------------------------------------------------------------ warm-start network
class UNetWarmStart:
    """The warm-start U-Net (wp_unet_*): predict(p, b, sdf, h) writes a multigrid starting guess,
    train_step(...) runs one Adam step on the GPU."""

    def __init__(self, dim, seed=0):
        self.dim = _dims3(dim)
        h = ctypes.c_void_p()
        check(lib().wp_unet_create(ctypes.byref(h), *self.dim, int(seed)), "wp_unet_create")
        self._h = h
        self.cells = mac_shapes3d(*self.dim)["p"]

    def predict(self, p, b, sdf, hcell, stream=None):
        c = self.cells
        check(lib().wp_unet_predict(self._h, _ptr(p, c), _ptr(b, c), _ptr(sdf, c), float(hcell), _stream(stream)),
              "wp_unet_predict")

    def train_step(self, b, sdf, p_target, hcell, lr, stream=None) -> float:
        c = self.cells
        loss = ctypes.c_double()
        check(lib().wp_unet_train_step(self._h, _ptr(b, c), _ptr(sdf, c), _ptr(p_target, c), float(hcell), float(lr),
                                       ctypes.byref(loss), _stream(stream)), "wp_unet_train_step")
        return loss.value

    def params(self, which=0):
        import numpy as np
        n = ctypes.c_size_t()
        check(lib().wp_unet_params(self._h, int(which), None, 0, ctypes.byref(n)), "wp_unet_params")
        out = np.empty(n.value, np.float32)
        check(lib().wp_unet_params(self._h, int(which), out.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n)),
              "wp_unet_params")
        return out

    def set_params(self, vec):
        import numpy as np
        v = np.ascontiguousarray(vec, np.float32)
        check(lib().wp_unet_set_params(self._h, v.ctypes.data_as(ctypes.c_void_p), v.size), "wp_unet_set_params")

    def close(self):
        if getattr(self, "_h", None):
            lib().wp_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
