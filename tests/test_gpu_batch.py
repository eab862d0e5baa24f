"""Batched projection of uneven 2D/3D grids in one CUDA graph (wp_batch_*), checked grid by grid
against the one-grid path (Projector3D / Projector2D, itself checked against the oracle) and, for
one 3D and one 2D grid, directly against the FP64 oracle's recovery of the projected field."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def T(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def N(t):
    return t.detach().double().cpu().numpy()


def rel(ref, got):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    return float(np.sqrt(np.sum((ref - got) ** 2) / max(np.sum(ref * ref), 1e-300)))


def _grids(wp):
    from waveletpotentials_b200 import fields
    specs = [(32, 32, 32), (256, 128), (16, 32, 64), (64, 64), (64, 32, 32), (128, 128), (32, 32, 32)]
    grids, u = [], []
    for i, d in enumerate(specs):
        h = 1.0 / d[0]
        nsph = i % 4
        c, r = fields.random_spheres(nsph, 0.05, 0.15, seed=100 + i)
        if len(d) == 3:
            s = wp.mac_shapes3d(*d)
            sls = wp.CuSolidLevelSet3D(d, h)
            sls.InitLsSpheres(c, r)
            a = [torch.empty(s[k], device="cuda") for k in ("xv", "yv", "zv")]
            sls.GetFrac(*a)
            grids.append({"dim": d, "dx": h, "ax": a[0], "ay": a[1], "az": a[2]})
            u.append([T(x) for x in fields.velocity3d(d, seed=200 + i)])
        else:
            s = wp.mac_shapes2d(*d)
            sls = wp.CuSolidLevelSet2D(d, h)
            sls.InitLsCircles(c[:, :2], r)
            a = [torch.empty(s[k], device="cuda") for k in ("xv", "yv")]
            sls.GetFrac(*a)
            grids.append({"dim": d, "dx": h, "ax": a[0], "ay": a[1]})
            u.append([T(x) for x in fields.velocity2d(d, seed=200 + i)])
    torch.cuda.synchronize()
    return grids, u


def _outs(wp, grids):
    outs = []
    for g in grids:
        d = g["dim"]
        if len(d) == 3:
            s = wp.mac_shapes3d(*d)
            outs.append([torch.full(s[k], 7.0, device="cuda") for k in ("qx", "qy", "qz")])
        else:
            outs.append([torch.full(wp.mac_shapes2d(*d)["qz"], 7.0, device="cuda")])
    return outs


@pytest.mark.parametrize("nstreams,start,inner", [(1, 0, 1), (4, 0, 1), (4, 1, 1), (4, 0, 3)])
def test_batch_matches_single_grid_path(wp, nstreams, start, inner):
    tol = 1e-9
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids, rel_tol=tol, max_cycles=40, nstreams=nstreams, start=start, inner_cycles=inner)
    cycles = bp.plan(u)
    assert all(1 <= c <= 40 for c in cycles)
    for rnd in range(2):  # the second run replays the captured graph on fresh copies of the fields
        fu = [[x.clone() for x in f] for f in u]
        outs = _outs(wp, grids)
        bp.run(fu, outs)
        res = bp.results()
        assert res["cycles"] == cycles
        for i, g in enumerate(grids):
            d = g["dim"]
            ref_u = [x.clone() for x in u[i]]
            if len(d) == 3:
                pr = wp.Projector3D(g["ax"], g["ay"], g["az"], d, g["dx"], rel_tol=tol, max_cycles=40, start=start,
                                    inner_cycles=inner)
                s = wp.mac_shapes3d(*d)
                ref_q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
                rep = pr.run(*ref_u, *ref_q)
            else:
                pr = wp.Projector2D(g["ax"], g["ay"], d, g["dx"], rel_tol=tol, max_cycles=40, start=start,
                                    inner_cycles=inner)
                ref_q = [torch.zeros(wp.mac_shapes2d(*d)["qz"], device="cuda")]
                rep = pr.run(*ref_u, *ref_q)
            assert rep["cycles"] == cycles[i], (i, rep["cycles"], cycles[i])
            assert res["rel_residual"][i] <= tol, (i, res["rel_residual"][i])
            assert abs(res["rel_residual"][i] - rep["rel_residual"]) <= 1e-2 * rep["rel_residual"] + 1e-14
            assert abs(res["max_abs_div"][i] - rep["max_abs_div"]) <= 1e-3 * max(rep["max_abs_div"], 1e-3), i
            for a, b in zip(ref_u, fu[i]):
                assert rel(N(a), N(b)) < 1e-6, (i, rnd)
            for a, b in zip(ref_q, outs[i]):
                assert rel(N(a), N(b)) < 1e-6, (i, rnd)


def test_batch_recovery_matches_oracle(wp, oracle):
    grids, u = _grids(wp)
    sel = [0, 1]  # one 3D and one 2D grid
    grids = [grids[i] for i in sel]
    u = [u[i] for i in sel]
    bp = wp.BatchProjector(grids, rel_tol=1e-8, max_cycles=40, nstreams=2)
    bp.plan(u)
    outs = _outs(wp, grids)
    bp.run(u, outs)
    torch.cuda.synchronize()
    d3 = grids[0]["dim"]
    h3 = grids[0]["dx"]
    oq = oracle.recover3d(*[N(t) for t in u[0]], d3, (h3,) * 3)
    for o, t in zip(oq, outs[0]):
        assert rel(o, N(t)) < TOL32
    d2 = grids[1]["dim"]
    h2 = grids[1]["dx"]
    oq2 = oracle.recover2d(*[N(t) for t in u[1]], d2, (h2,) * 2)
    assert rel(oq2, N(outs[1][0])) < TOL32
    # the projected (fraction-weighted) field is discretely divergence-free to the solve tolerance
    res = bp.results()
    b = oracle.divergence3d(*[N(t) for t in u[0]], *[np.ones_like(N(t)) for t in u[0]], d3, (h3,) * 3)
    assert abs(np.max(np.abs(b)) - res["max_abs_div"][0]) <= 1e-2 * max(1.0, res["max_abs_div"][0])


def test_batch_rejects_bad_arguments(wp):
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids[:2], rel_tol=1e-6, nstreams=2)
    outs = _outs(wp, grids[:2])
    with pytest.raises(wp.WPError):
        bp.run([[u[0][0], u[0][1], torch.zeros(3, device="cuda")], u[1]], outs)  # a 3D grid's zv of a wrong shape
    s = wp.mac_shapes2d(48, 64)  # 48 is not a power of two: the wavelet recovery rejects it
    bad = {"dim": (48, 64), "dx": 1 / 64, "ax": torch.ones(s["xv"], device="cuda"),
           "ay": torch.ones(s["yv"], device="cuda")}
    with pytest.raises(wp.WPError):
        wp.BatchProjector([bad], rel_tol=1e-6)


def test_sharded_batch_shares_match_whole_batch(wp):
    """The batch split by cost into two shares (both built here on one GPU, as two ranks would build
    theirs): every grid lands in exactly one share, and each share's per-grid results and projected
    fields equal those of the whole batch run as one."""
    from waveletpotentials_b200 import sharding
    tol = 1e-8
    grids, u = _grids(wp)
    whole = wp.BatchProjector(grids, rel_tol=tol, max_cycles=40, nstreams=4)
    cycles = whole.plan(u)
    fw = [[x.clone() for x in f] for f in u]
    ow = _outs(wp, grids)
    whole.run(fw, ow)
    rw = whole.results()
    shares = [sharding.ShardedBatch(grids, rank=r, world=2, rel_tol=tol, steps=cycles, max_cycles=40, nstreams=4)
              for r in range(2)]
    assert sorted(shares[0].mine + shares[1].mine) == list(range(len(grids)))
    assert shares[0].owner == shares[1].owner
    local = {}
    for sh in shares:
        fs = [[x.clone() for x in u[i]] for i in sh.mine]
        os_ = [_outs(wp, [grids[i]])[0] for i in sh.mine]
        assert sh.plan([u[i] for i in sh.mine]) == [cycles[i] for i in sh.mine]
        sh.run(fs, os_)
        local.update(sh.local_results())
        for k, i in enumerate(sh.mine):
            for a, b in zip(ow[i], os_[k]):
                assert rel(N(a), N(b)) < 1e-6, i
    merged = sharding.gather_results(local, len(grids), 1)
    for i, m in enumerate(merged):
        assert m["cycles"] == rw["cycles"][i] and m["over_tol"] is False
        assert abs(m["rel_residual"] - rw["rel_residual"][i]) <= 1e-2 * rw["rel_residual"][i] + 1e-14
    for sh in shares:
        sh.close()
