"""Persistent batched solve (wp_batch_set_mode(..., WP_BATCH_PERSISTENT)): every grid's mixed-precision
solve in one persistent kernel that takes (grid, level, pass) tiles from a device work queue, checked
against the graph batch (each grid's solve its own device loop of launches, itself checked against
the one-grid path in test_gpu_batch.py) on uneven 2D/3D grids with solids: the same V-cycle counts,
the same projected fields and potentials, on replays and for several tile sizes; the cycle cap, a
withheld publication (the kernel's bounded waits give up and the batch stays usable), and the
configurations the persistent program does not take."""
import pytest
import torch

from test_gpu_batch import N, _grids, _outs, rel

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _clone(u):
    return [[x.clone() for x in f] for f in u]


def _run(bp, u, grids, wp):
    fu = _clone(u)
    outs = _outs(wp, grids)
    bp.run(fu, outs)
    return fu, outs, bp.results()


# FP32 parity tolerance (relative L2): the two paths agree to rounding, and on grids whose projected
# field is near zero (potentials of 1e-9) rounding alone is 1e-6 of it
TOL32 = 1e-5


def _same_fields(a_u, a_q, b_u, b_q, tol=TOL32):
    for i in range(len(a_u)):
        for x, y in zip(a_u[i], b_u[i]):
            assert rel(N(x), N(y)) < tol, i
        for x, y in zip(a_q[i], b_q[i]):
            assert rel(N(x), N(y)) < tol, i


@pytest.mark.parametrize("inner,tile_cells", [(1, 0), (3, 0), (1, 4096), (1, 1 << 20)])
def test_persistent_batch_matches_graph_batch(wp, inner, tile_cells):
    grids, u = _grids(wp)
    ref = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=4, inner_cycles=inner)
    cycles = ref.plan(u)
    ru, rq, rres = _run(ref, u, grids, wp)
    assert rres["status"] == "WP_OK" and rres["cycles"] == cycles
    bp = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=4, inner_cycles=inner, persistent=True,
                           tile_cells=tile_cells)
    assert bp.mode == wp.BATCH_PERSISTENT
    assert bp.plan(u) == cycles
    for rnd in range(2):  # the second run replays the captured graph: the queue state is set up again
        pu, pq, res = _run(bp, u, grids, wp)
        assert res["status"] == "WP_OK", (rnd, res)
        assert res["cycles"] == cycles, (rnd, res["cycles"], cycles)
        _same_fields(ru, rq, pu, pq)
        for i in range(len(grids)):
            assert res["rel_residual"][i] <= TOL, (i, res["rel_residual"][i])
            assert abs(res["rel_residual"][i] - rres["rel_residual"][i]) <= 1e-2 * rres["rel_residual"][i] + 1e-14
            # max|div u| of an FP32 field after a 1e-9 solve is the largest FP32 rounding residue over the
            # cells; iterates that differ in the last bits (the FP64 mean and norms are summed in another
            # order) give another draw of that residue, of the same size
            a, b = res["max_abs_div"][i], rres["max_abs_div"][i]
            assert a <= 2.0 * b + 1e-9 and b <= 2.0 * a + 1e-9, (i, a, b)


def test_persistent_batch_without_plan_and_mode_switch(wp):
    """No plan: the programs are ordered by size.  Switching back to the graph mode gives the same
    results."""
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=2, persistent=True)
    pu, pq, res = _run(bp, u, grids, wp)
    assert res["status"] == "WP_OK" and all(c >= 1 for c in res["cycles"]), res
    bp.set_mode(wp.BATCH_GRAPH)
    gu, gq, gres = _run(bp, u, grids, wp)
    assert gres["cycles"] == res["cycles"]
    _same_fields(gu, gq, pu, pq)


def test_persistent_tile_is_tuned_by_the_plan(wp):
    """With tile_cells 0 the plan times the persistent solve with each candidate tile and keeps the
    fastest; a tile the caller gives is kept as given."""
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids, rel_tol=1e-6, max_cycles=40, nstreams=2, persistent=True)
    assert bp.get_mode()[0] == wp.BATCH_PERSISTENT
    bp.plan(u)
    mode, tile, ms, graph_ms = bp.get_mode()
    cands = wp.BatchProjector.TILE_CANDIDATES
    assert mode == wp.BATCH_PERSISTENT and tile in cands, (tile, ms)
    assert len(ms) == len(cands) and all(t > 0 for t in ms) and ms[cands.index(tile)] == min(ms), ms
    _, _, res = _run(bp, u, grids, wp)
    assert res["status"] == "WP_OK"
    fixed = wp.BatchProjector(grids, rel_tol=1e-6, max_cycles=40, nstreams=2, persistent=True, tile_cells=4096)
    fixed.plan(u)
    assert fixed.get_mode()[1] == 4096 and fixed.get_mode()[2] == [0.0] * len(cands)


@pytest.mark.parametrize("which", ["small", "mixed"])
def test_auto_mode_runs_the_faster_way(wp, which):
    """BATCH_AUTO: the plan times the persistent solve (tile tuned) and the graph mode's solves on its
    inputs and runs the faster one; before a plan it runs as a graph.  The results equal the graph
    mode's either way."""
    grids, u = _grids(wp)
    if which == "small":
        keep = [i for i, g in enumerate(grids) if len(g["dim"]) == 3 and max(g["dim"]) <= 32 or
                len(g["dim"]) == 2 and max(g["dim"]) <= 64]
        grids, u = [grids[i] for i in keep], [u[i] for i in keep]
    bp = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=2, mode=wp.BATCH_AUTO)
    assert bp.get_mode()[0] == wp.BATCH_GRAPH
    cycles = bp.plan(u)
    mode, tile, ms, graph_ms = bp.get_mode()
    assert graph_ms > 0 and min(ms) > 0, (ms, graph_ms)
    pers_ms = ms[wp.BatchProjector.TILE_CANDIDATES.index(tile)]
    assert mode == (wp.BATCH_PERSISTENT if pers_ms < graph_ms else wp.BATCH_GRAPH), (mode, pers_ms, graph_ms)
    au, aq, res = _run(bp, u, grids, wp)
    assert res["status"] == "WP_OK" and res["cycles"] == cycles, res
    ref = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=2)
    ref.plan(u)
    gu, gq, gres = _run(ref, u, grids, wp)
    assert gres["cycles"] == res["cycles"]
    _same_fields(gu, gq, au, aq)


def test_persistent_batch_cycle_cap(wp):
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids, rel_tol=1e-12, max_cycles=2, nstreams=2, persistent=True)
    _, _, res = _run(bp, u, grids, wp)
    assert res["status"] == "WP_ERR_NOT_CONVERGED" and all(res["over_tol"]), res
    assert res["cycles"] == [2] * len(grids), res


def test_persistent_batch_withheld_publication(wp):
    """The phase after phase 2 of the first grid is never published: every CTA then finds no work
    until its bounded wait (50 ms here) runs out; the grids still running report it, the launch ends,
    wp_batch_results returns WP_ERR_DEVICE_WAIT, and the next run of the same batch gives the
    undisturbed results."""
    grids, u = _grids(wp)
    bp = wp.BatchProjector(grids, rel_tol=TOL, max_cycles=40, nstreams=2, persistent=True)
    ou, oq, ores = _run(bp, u, grids, wp)
    assert ores["status"] == "WP_OK"
    wp.debug_withhold_wait(wp.WAIT_SITE_BATCH_PUBLISH, at=2, limit_s=0.05)
    bp.run(_clone(u), _outs(wp, grids))
    with pytest.raises(wp.WPError) as ei:
        bp.results()
    assert ei.value.status == wp._lib.WP_ERR_DEVICE_WAIT
    pu, pq, res = _run(bp, u, grids, wp)
    assert res["status"] == "WP_OK" and res["cycles"] == ores["cycles"], res
    _same_fields(ou, oq, pu, pq)


def test_persistent_batch_refuses_what_it_does_not_run(wp):
    """Piecewise-constant prolongation and a full-multigrid start are not programs of the persistent
    kernel: the mode switch fails with WP_ERR_UNSUPPORTED and the batch keeps running as a graph (the
    piecewise-constant cycle, the reference's, need not reach the tolerance: its run only has to end
    with every grid's results)."""
    grids, u = _grids(wp)
    grids, u = grids[:2], u[:2]
    for kw in ({"prolongation": wp.PROLONG_CONSTANT}, {"start": wp.START_FMG}):
        bp = wp.BatchProjector(grids, rel_tol=1e-6, max_cycles=40, nstreams=2, **kw)
        with pytest.raises(wp.WPError) as ei:
            bp.set_mode(wp.BATCH_PERSISTENT)
        assert ei.value.status == 2  # WP_ERR_UNSUPPORTED
        _, _, res = _run(bp, u, grids, wp)
        ok = ("WP_OK", "WP_ERR_NOT_CONVERGED") if "prolongation" in kw else ("WP_OK",)
        assert res["status"] in ok and all(c >= 1 for c in res["cycles"]), (kw, res)
    bp = wp.BatchProjector(grids, rel_tol=1e-6, max_cycles=40, nstreams=2)
    with pytest.raises(wp.WPError):
        bp.set_mode(7)
    with pytest.raises(wp.WPError):
        bp.set_mode(wp.BATCH_PERSISTENT, -1)
