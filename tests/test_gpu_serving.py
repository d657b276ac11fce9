"""Serving form (afsi_gpu_b200.serving): continuous batching over resident states.

A request's result must not depend on what else runs: in the mix and alone,
pressure solves and interpolated velocities are bitwise equal (deterministic
kernels, same inputs), spread fields equal to 1e-12 of their scale (the
spread's L2 atomics may add in another order).
"""
import pytest
import torch
from afsi_gpu_b200.serving import Request, Server, mix, request_bytes

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def test_results_in_the_mix_equal_results_alone():
    reqs = mix(24, rate=2000., seed=3, scale=.05)
    server = Server(device=DEV, slots=4, keep_results=True)
    report, results = server.serve(reqs)
    assert report['requests'] == len(reqs) and len(results) == len(reqs)
    assert 0 < report['p50_ms'] <= report['p99_ms'] and report['steps_per_s'] > 0
    kinds = {}
    for r in reqs:
        kinds.setdefault((r.kind, r.n), r)
    for req in kinds.values():
        alone = server.alone(req)
        mixed = results[req.rid]
        assert torch.equal(alone['pressure'], mixed['pressure'])
        assert alone['cycles'] == mixed['cycles']
        assert torch.equal(alone['velocity'], mixed['velocity'])
        for a, m in zip(alone['fields'], mixed['fields']):
            scale = a.abs().max().item()
            assert (a - m).abs().max().item() <= 1e-12 * scale


def test_admission_respects_the_hbm_budget():
    """With room for the resident states and one request, three slots still
    serve every request, one at a time; a budget below the resident states is
    refused up front."""
    reqs = [Request(0., i, '2d', 256, 4000, seed=i) for i in range(6)]
    one = Server(device=DEV, slots=1)
    one.warm(reqs)
    need = request_bytes(reqs[0])
    server = Server(device=DEV, slots=3, budget_bytes=3 * one.resident + need + 1)
    report, _ = server.serve(reqs)
    assert report['requests'] == len(reqs) and report['peak_request_bytes'] == need
    with pytest.raises(MemoryError):
        Server(device=DEV, slots=1, budget_bytes=10).serve(reqs)
