"""C ABI surface (no GPU needed): the in-tree library builds, loads, exports every entry point
include/wp_api.h declares, and rejects invalid arguments with a status code before touching CUDA."""
import ctypes

import pytest

from waveletpotentials_b200 import _lib, build


@pytest.fixture(scope="module")
def L():
    build.build()
    return _lib.lib()


def test_every_declared_symbol_is_exported(L):
    names = _lib.header_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_version_and_error_string(L):
    assert L.wp_version() >= 1
    assert isinstance(_lib.last_error(), str)


def _c(ch):
    return ctypes.c_char(ch.encode())


def test_dwt_rejects_bad_shapes(L):
    dummy = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    # line length 20 is not 2^levels (+1)
    assert L.wp_dwt1d(dummy, dummy, 20, 4, 4, 4, _c("x"), _c("n"), _lib.CDF3_7, 1, None) == 1
    assert "2^levels" in _lib.last_error()
    assert L.wp_dwt1d(dummy, dummy, 16, 4, 4, 4, _c("w"), _c("n"), _lib.CDF3_7, 1, None) == 1
    assert L.wp_dwt1d(dummy, dummy, 16, 4, 4, 4, _c("x"), _c("q"), _lib.CDF3_7, 1, None) == 1
    assert L.wp_dwt1d(dummy, dummy, 16, 4, 4, 4, _c("x"), _c("n"), 3, 1, None) == 2  # CDF2.10: another family
    assert L.wp_dwt1d(None, None, 16, 4, 4, 4, _c("x"), _c("n"), _lib.CDF3_7, 1, None) == 1
    # the short families register 'n' and 'd' only
    for wav in (_lib.CDF2_0, _lib.CDF1_1, _lib.CDF1_7):
        assert L.wp_dwt1d(dummy, dummy, 16, 4, 4, 4, _c("x"), _c("z"), wav, 1, None) == 1
        assert "take bc 'n' or 'd'" in _lib.last_error()


def test_recover_rejects_unsupported_requests(L):
    h = ctypes.c_void_p()
    assert L.wp_recover3d_create(ctypes.byref(h), 24, 16, 16, 0.1, 0.1, 0.1, _c("n"), 11, 7) == 1
    assert L.wp_recover3d_create(ctypes.byref(h), 16, 16, 16, 0.1, 0.1, 0.1, _c("z"), 11, 7) == 2
    assert "bc must be 'n'" in _lib.last_error()
    assert L.wp_recover3d_create(ctypes.byref(h), 16, 16, 16, 0.1, 0.1, 0.1, _c("n"), 7, 11) == 2
    assert L.wp_recover3d_create(ctypes.byref(h), 16, 16, 16, 0.0, 0.1, 0.1, _c("n"), 11, 7) == 1
    assert L.wp_recover2d_create(ctypes.byref(h), 16, 12, 0.1, 0.1, _c("n"), 11, 7) == 1
    assert L.wp_recover3d_run(None, None, None, None, None, None, None, None) == 1


def test_multigrid_rejects_bad_arguments(L):
    h = ctypes.c_void_p()
    dummy = ctypes.c_void_p(16)
    assert L.wp_mgfrac3d_create(ctypes.byref(h), None, dummy, dummy, 8, 8, 8, 0.1, 0.1, 0.1, _c("n"), None) == 1
    assert L.wp_mgfrac3d_create(ctypes.byref(h), dummy, dummy, dummy, 8, 8, 8, 0.1, 0.1, 0.1, _c("d"), None) == 2
    assert L.wp_mgfrac3d_create(ctypes.byref(h), dummy, dummy, dummy, 1, 8, 8, 0.1, 0.1, 0.1, _c("n"), None) == 1
    assert L.wp_mgfrac3d_solve(None, dummy, None, dummy, 3, 2, 2, 0.8, None) == 1
    prm = _lib.MgParams(10, 2, 2, 0.8, 1e-6, 7, 1)
    assert L.wp_mgfrac3d_solve_tol(None, dummy, None, dummy, ctypes.byref(prm), None, None) == 1
    assert L.wp_mgfrac2d_solve(None, dummy, None, dummy, 3, 2, 2, 0.8, None) == 1
    assert L.wp_mgfrac3d_solve_index(None, dummy, None, dummy, 3, 2, 2, 0.8, None) == 1
    assert L.wp_mgfrac3d_index_sizes(None, None, None, 4, None, None) == 1


def test_field_operators_reject_bad_arguments(L):
    dummy = ctypes.c_void_p(16)
    assert L.wp_divergence_frac3d(None, dummy, dummy, dummy, dummy, dummy, dummy, 4, 4, 4, 1., 1., 1., None) == 1
    # a partial set of fraction pointers is an error (all NULL means open faces)
    assert L.wp_divergence_frac3d(dummy, dummy, dummy, dummy, dummy, None, None, 4, 4, 4, 1., 1., 1., None) == 1
    assert L.wp_grad_subtract_frac3d(dummy, dummy, dummy, None, dummy, dummy, dummy, 4, 4, 4, 1., 1., 1., 1,
                                     None) == 1
    out = ctypes.c_double()
    assert L.wp_max_abs(None, 10, ctypes.byref(out), None) == 1
    assert L.wp_sdf_spheres3d(dummy, 4, 4, 4, 0.25, None, None, 2, None) == 1
