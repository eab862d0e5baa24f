"""HostPipeline3D: projections of host-resident fields with overlapped transfers give the results of
Projector3D.run step by step."""
import numpy as np
import pytest
import torch

from test_gpu_parity import _sphere_problem

pytestmark = pytest.mark.gpu


def test_host_pipeline_matches_one_by_one(wp, oracle):
    from waveletpotentials_b200 import fields
    nn, h, a, _, _ = _sphere_problem(wp, oracle, 32, seed=2)
    ta = [torch.as_tensor(x, dtype=torch.float32, device="cuda") for x in a]
    s = wp.mac_shapes3d(*nn)
    inputs = [tuple(np.asarray(x, dtype=np.float32) for x in fields.velocity3d(nn, 40 + k)) for k in range(5)]
    # one by one through Projector3D.run
    ref = []
    pr = wp.Projector3D(*ta, nn, h, rel_tol=1e-10, precision=wp.PREC_MIXED)
    for u in inputs:
        tu = [torch.as_tensor(x, device="cuda") for x in u]
        q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
        rep = pr.run(*tu, *q)
        ref.append((rep, [t.cpu().numpy() for t in q]))
    # the same fields through the pipeline, from pinned host memory into pinned host memory
    pipe = wp.HostPipeline3D(wp.Projector3D(*ta, nn, h, rel_tol=1e-10, precision=wp.PREC_MIXED))
    host_in = [[torch.from_numpy(x).pin_memory() for x in u] for u in inputs]
    host_out = [[torch.zeros(s[k], dtype=torch.float32).pin_memory() for k in ("qx", "qy", "qz")] for _ in inputs]
    reps = pipe.run(host_in, host_out)
    assert pipe.h2d_bytes == sum(x.nbytes for x in inputs[0])
    for (rrep, rq), rep, hq in zip(ref, reps, host_out):
        assert rep["status"] == "WP_OK" and rep["cycles"] == rrep["cycles"]
        for got, want in zip(hq, rq):
            scale = np.abs(want).max()
            assert np.abs(got.numpy() - want).max() <= 1e-5 * scale
    # inputs on the host are untouched (the projection works on the device copies)
    for u, hu in zip(inputs, host_in):
        for x, t in zip(u, hu):
            assert np.array_equal(x, t.numpy())
