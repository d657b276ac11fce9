"""Host logic of the serving and batching forms (no GPU).

The serving mix: the configured shares of request kinds (50 % 2D 256x64 with
20k points, 35 % 3D 32^3-64^3 with 50k-400k points, 15 % 3D 96^3 with 800k
points) and Poisson arrivals at the configured rate, seeded; the admission's
HBM estimate grows with the request.  The batching workload: the leaflet
points of every instance lie inside the region the batched prepare accepts
(x in [2h, Lx - 2h], y in [-h, Ly + h]), so the seeded batch never trips the
support check.  Both forms refuse a CPU device: there is no CPU fallback.
"""
import numpy as np
import pytest
from afsi_gpu_b200.batch import leaflet_points
from afsi_gpu_b200.grid import ChannelGrid
from afsi_gpu_b200.serving import Request, Server, mix, request_bytes


def test_serving_mix_shares_and_poisson_arrivals():
    reqs = mix(4000, rate=2000., seed=0)
    kinds = np.array([(r.kind, r.n) for r in reqs], dtype=object)
    share_2d = np.mean([k == '2d' for k, _ in kinds])
    share_96 = np.mean([k == '3d' and n == 96 for k, n in kinds])
    share_mid = np.mean([k == '3d' and n in (32, 48, 64) for k, n in kinds])
    assert abs(share_2d - .50) < .03 and abs(share_mid - .35) < .03 and abs(share_96 - .15) < .03
    t = np.array([r.arrival for r in reqs])
    gaps = np.diff(np.concatenate(([0.], t)))
    assert np.all(gaps > 0)
    assert abs(gaps.mean() * 2000. - 1.) < .05          # mean inter-arrival 1/rate
    assert abs(gaps.std() / gaps.mean() - 1.) < .08     # exponential: coefficient of variation 1
    for r in reqs:
        if r.kind == '2d':
            assert (r.n, r.points) == (256, 20000)
        elif r.n == 96:
            assert r.points == 800000
        else:
            assert 50000 <= r.points <= 400000
    assert [r.rid for r in mix(50, seed=3)] == list(range(50))
    assert [r.points for r in mix(50, seed=3)] == [r.points for r in mix(50, seed=3)]


def test_admission_estimate_grows_with_the_request():
    small = request_bytes(Request(0., 0, '3d', 32, 50000, 0))
    more_points = request_bytes(Request(0., 0, '3d', 32, 400000, 0))
    bigger_grid = request_bytes(Request(0., 0, '3d', 96, 50000, 0))
    assert 0 < small < more_points and small < bigger_grid
    assert request_bytes(Request(0., 0, '2d', 256, 20000, 0)) > 0


@pytest.mark.parametrize('shape', [(128, 32), (256, 64), (384, 96), (512, 128)])
def test_leaflet_points_lie_inside_the_batched_support_region(shape):
    g = ChannelGrid(shape, (4., 1.))
    hx, hy = g.spacing
    for seed in range(5):
        p = leaflet_points(g, 40000, seed)
        assert p.shape == (40000, 2)
        assert np.all(p[:, 0] >= 2 * hx) and np.all(p[:, 0] <= g.lengths[0] - 2 * hx)
        assert np.all(p[:, 1] >= -hy) and np.all(p[:, 1] <= g.lengths[1] + hy)


def test_forms_refuse_a_cpu_device():
    with pytest.raises(ValueError, match='CUDA'):
        Server(device='cpu')


def test_request_inputs_are_made_once_and_seeded():
    """Request inputs are host tensors made from the seed (the serving clock
    never includes their generation): point and force shapes per kind, a
    mean-free pressure right-hand side on the request's grid."""
    from afsi_gpu_b200.serving import make_inputs, grid_of
    for req in (Request(0., 0, '2d', 256, 3000, 7), Request(0., 1, '3d', 32, 2000, 8)):
        a, b = make_inputs(req, pin=False), make_inputs(req, pin=False)
        d = 2 if req.kind == '2d' else 3
        assert a['points'].shape == (req.points, d) and a['force'].shape == (req.points, d)
        assert tuple(a['rhs'].shape) == tuple(grid_of(req.kind, req.n).shape)
        assert abs(float(a['rhs'].mean())) < 1e-12
        assert all(np.array_equal(a[k].numpy(), b[k].numpy()) for k in a)
