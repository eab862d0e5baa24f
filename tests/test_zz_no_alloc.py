"""Allocation-free DST-I solve (wp_dst3d_solve_noalloc) against the handle-based entry point
(wp_dst3d_create + wp_dst3d_solve) and the FP64 oracle, on two calls in a row.  Kept in its own
file, named to be collected last, so it also runs after every other GPU test in the session."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


def test_noalloc_dst_matches_handle_path_on_consecutive_calls(wp, oracle):
    rng = np.random.default_rng(404)
    cases = [((24, 20, 16), (1 / 25, 1 / 21, 1 / 17)), ((64, 64, 64), (1 / 64, 1 / 64, 1 / 64))]
    for n, h in cases:
        # two calls in a row on different right-hand sides: the second must not see the first's state
        fs = [rng.standard_normal((n[2], n[0], n[1])) for _ in range(2)]
        handle = wp.CuDst3D(n, h)
        for f in fs:
            ft = torch.as_tensor(f, dtype=torch.float64, device="cuda")
            want = torch.empty_like(ft)
            handle.Solve(want, ft)
            got = torch.full_like(ft, float("nan"))
            wp.CuDst3D.SolveNoAlloc(got, ft, n, h)
            torch.cuda.synchronize()
            assert rel(want.cpu().numpy(), got.cpu().numpy()) < 1e-13
            if n[0] <= 32:
                assert rel(oracle.dst3d_poisson(f, n, h), got.cpu().numpy()) < 1e-12
        handle.close()


def test_noalloc_dst_in_place_and_size_limit(wp):
    n, h = (32, 16, 8), (1 / 33, 1 / 17, 1 / 9)
    f = torch.as_tensor(np.random.default_rng(5).standard_normal((n[2], n[0], n[1])), dtype=torch.float64,
                        device="cuda")
    want = torch.empty_like(f)
    wp.CuDst3D(n, h).Solve(want, f)
    g = f.clone()
    wp.CuDst3D.SolveNoAlloc(g, g, n, h)
    torch.cuda.synchronize()
    assert rel(want.cpu().numpy(), g.cpu().numpy()) < 1e-13
    # beyond the static scratch: rejected on the host with a clear message, nothing launched
    big = torch.zeros((4, 65, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(wp.WPError, match="static scratch"):
        wp.CuDst3D.SolveNoAlloc(big, big, (65, 8, 4), 1 / 65)
