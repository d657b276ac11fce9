"""Serving form (afsi_gpu_b200.serving): continuous batching over resident states.

A request's result must not depend on what else runs.  In the mix and alone:
interpolated velocities are bitwise equal (per-point arithmetic, same
inputs); spread fields equal to 1e-12 of their scale (the spread's atomic
additions may land in another order); FP64 pressures bitwise equal; pressures
of the FP32-refined form (batched refinement runs until every instance of a
batch meets its tolerance, so an instance may get another refinement) within
1e-8 of their scale, every one at the 1e-10 relative residual.
"""
import numpy as np
import pytest
import torch
from afsi_gpu_b200.serving import Request, Server, mix, request_bytes, with_inputs

pytestmark = pytest.mark.gpu
DEV = 'cuda'


@pytest.mark.parametrize('precision', ['fp64', 'fp32-refined'])
def test_results_in_the_mix_equal_results_alone(precision):
    reqs = with_inputs(mix(24, rate=20000., seed=3, scale=.05))
    server = Server(device=DEV, slots=3, batch=4, keep_results=True, precision=precision)
    report, results = server.serve(reqs)
    assert report['requests'] == len(reqs) and len(results) == len(reqs)
    assert 0 < report['p50_ms'] <= report['p99_ms'] and report['steps_per_s'] > 0
    assert report['batches_2d']['max_size'] > 1  # requests that arrived together were batched
    kinds = {}
    for r in reqs:
        kinds.setdefault((r.kind, r.n), r)
    for req in kinds.values():
        alone = server.alone(req)
        mixed = results[req.rid]
        assert torch.equal(alone['velocity'], mixed['velocity'])
        for a, m in zip(alone['fields'], mixed['fields']):
            assert (a - m).abs().max().item() <= 1e-12 * a.abs().max().item()
        pa, pm = alone['pressure'], mixed['pressure']
        if precision == 'fp64' or req.kind == '3d':
            assert torch.equal(pa, pm)
        else:
            assert (pa - pm).abs().max().item() <= 1e-8 * pa.abs().max().item()


def test_refined_batches_meet_the_fp64_tolerance():
    """Every 2D pressure served by the batched refinement meets the FP64
    solver's relative residual 1e-10 (checked with the FP64 operator)."""
    from oracle import mg as omg
    from afsi_gpu_b200.serving import grid_of
    reqs = with_inputs([Request(0., i, '2d', 256, 3000, seed=40 + i) for i in range(5)])
    server = Server(device=DEV, slots=1, batch=5, keep_results=True, precision='fp32-refined')
    report, results = server.serve(reqs)
    assert report['batches_2d']['max_size'] >= 2
    g = grid_of('2d', 256)
    h = omg.Hierarchy(g.shape, g.spacing, 'channel')
    for r in reqs:
        b = r.inputs['rhs'].numpy()
        p = results[r.rid]['pressure'].numpy()
        assert np.linalg.norm(b - h.apply(0, p)) <= 1e-10 * np.linalg.norm(b)


def test_admission_respects_the_hbm_budget():
    """With room for the resident states and one request, every request is
    still served, one at a time; a budget below the resident states is
    refused up front."""
    reqs = with_inputs([Request(0., i, '3d', 32, 4000, seed=i) for i in range(6)])
    server = Server(device=DEV, slots=3, batch=2)
    server.warm(reqs)
    need = request_bytes(reqs[0])
    server.budget = server.resident + need + 1
    report, _ = server.serve(reqs)
    assert report['requests'] == len(reqs) and report['peak_request_bytes'] == need
    with pytest.raises(MemoryError):
        Server(device=DEV, slots=1, budget_bytes=10).serve(reqs)
