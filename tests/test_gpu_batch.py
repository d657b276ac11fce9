"""Batching form (afsi_gpu_b200.batch): many 2D channel instances per step.

Per instance the batch must reproduce the single-instance operators: stencil
ids and FP64 weights bit-exact against the oracle (``mac2d/transfer.py:61-81``),
FP32 weights equal to the FP64 weights rounded once; spreads and gathers
1e-12 of the field scale in FP64 (the single-instance bar) and 2e-6 in FP32
against the FP64 oracle; each instance's V-cycles, per instance over streams or batched
(one launch per level operation for all instances), bitwise equal to its own
solver run alone; graph replay equal to the eager step.
"""
import numpy as np
import pytest
import torch
from oracle import ib as oracle
from afsi_gpu_b200.batch import Schedule, seeded_batch

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def _small(dtype, count=6, seed=4, vcycles='streams'):
    return seeded_batch(count, seed=seed, shapes=((128, 32), (256, 64), (384, 96), (512, 128), (32, 8)),
                        points=(2000, 6000), device=DEV, transfer_dtype=dtype,
                        schedule=Schedule(streams=3, order='largest-first', smoother='jacobi', cycles=3,
                                          vcycles=vcycles))


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_batched_transfers_match_oracle_per_instance(dtype):
    b = _small(dtype)
    b.run()
    torch.cuda.synchronize()
    b.check()
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    for i, g in enumerate(b.grids):
        lo, hi = b.point_offsets[i], b.point_offsets[i + 1]
        pts = b.x[lo:hi].cpu().numpy()
        ids, w = oracle.prepare2d(pts, g.shape, g.spacing)
        for c, off in enumerate((b.u_offsets[i], b.v_offsets[i])):
            assert np.array_equal(b.ids[c, lo:hi].cpu().numpy(), ids[c] + off)
            got_w = b.weights[c, lo:hi].cpu().numpy()
            assert np.array_equal(got_w, w[c].astype(got_w.dtype))
        force = b.force[lo:hi].double().cpu().numpy()
        fields = b.fields(i)
        vel = (b.u_in[b.u_offsets[i]:b.u_offsets[i + 1]], b.v_in[b.v_offsets[i]:b.v_offsets[i + 1]])
        for c in range(2):
            size = fields[c].numel()
            ref = oracle.indexed_spread(force[:, c], ids[c], w[c], size, g.volume)
            scale = np.abs(ref).max()
            np.testing.assert_allclose(fields[c].reshape(-1).double().cpu().numpy(), ref, rtol=tol, atol=tol * scale)
            ref = oracle.indexed_gather(vel[c].double().cpu().numpy(), ids[c], w[c])
            np.testing.assert_allclose(b.velocities(i)[:, c].double().cpu().numpy(), ref, rtol=tol,
                                       atol=tol * np.abs(ref).max())


@pytest.mark.parametrize('vcycles', ['streams', 'batched', 'persistent'])
def test_batched_cycles_equal_each_instance_alone_and_graph_replay_equals_eager(vcycles):
    b = _small(torch.float32, count=9, vcycles=vcycles)
    sch = b.schedule
    b.run(sch)
    torch.cuda.synchronize()
    eager_p = [b.pressure(i).clone() for i in range(len(b.grids))]
    eager_g = b.gathered.clone()
    from afsi_gpu_b200.multigrid import ChannelMultigrid, MGOptions
    for i, g in enumerate(b.grids):
        alone = ChannelMultigrid(g, device=DEV, dtype=torch.float32, coarse_dtype=torch.float64, backend='b200',
                                 options=MGOptions(smooth=4))
        alone.initialize(torch.zeros_like(eager_p[i]), b.rhs[i])
        p = alone.advance(sch.cycles)
        assert torch.equal(p, eager_p[i])
    reduction = b.residual_reduction()
    assert max(reduction) < 1e-2
    b.use(sch)  # captures (and so runs the step once more)
    for i in range(len(b.grids)):
        b.pressure(i).zero_()
    b.gathered.zero_()
    b.replay()
    torch.cuda.synchronize()
    b.check()
    assert torch.equal(b.gathered, eager_g)
    for i in range(len(b.grids)):
        assert torch.equal(b.pressure(i), eager_p[i])


def test_autotuner_picks_a_measured_schedule_meeting_the_target():
    b = _small(torch.float32, count=8, seed=7)
    schedule, table = b.autotune(target=1e-3, streams=(1, 4), max_cycles=10, replays=2)
    best = min(table, key=lambda r: r['ms'])
    assert (best['streams'], best['order'], best['smoother'], best['cycles']) == \
        (schedule.streams, schedule.order, schedule.smoother, schedule.cycles)
    assert {r['smoother'] for r in table} == {'jacobi', 'red-black'}
    assert {r['vcycles'] for r in table} == {'streams', 'batched', 'persistent'}
    b.replay()
    torch.cuda.synchronize()
    assert max(b.residual_reduction()) <= 1e-3


def test_batch_rejects_points_outside_their_channel():
    b = _small(torch.float64, count=2)
    b.x[0, 0] = -1.0
    b.run()
    with pytest.raises(ValueError, match='support'):
        b.check()


@pytest.mark.parametrize('persistent', [False, True])
@pytest.mark.parametrize('smooth', [3, 4])
def test_batched_vcycles_match_each_solver_alone(smooth, persistent):
    """Uneven grids (some wholly in one CTA, some with two launched levels),
    an odd and an even sweep count; a started run then a continued one."""
    from afsi_gpu_b200.batch import BatchedVCycles
    from afsi_gpu_b200.grid import ChannelGrid
    from afsi_gpu_b200.multigrid import ChannelMultigrid, MGOptions
    shapes = [(512, 128), (64, 16), (256, 64), (32, 8), (384, 96)]
    rng = np.random.default_rng(11)
    grids = [ChannelGrid(s, (4., 1.)) for s in shapes]

    def solver(g):
        return ChannelMultigrid(g, device=DEV, dtype=torch.float32, coarse_dtype=torch.float64, backend='b200',
                                options=MGOptions(smooth=smooth))
    rhs = [torch.as_tensor(rng.standard_normal(s), dtype=torch.float32, device=DEV) for s in shapes]
    batch = [solver(g) for g in grids]
    for mg in batch:
        mg.workspace.p[0].fill_(7.)   # the start must zero it
    bv = BatchedVCycles(batch, rhs)
    bv.run(2, persistent=persistent)
    bv.run(1, start=False, persistent=persistent)
    torch.cuda.synchronize()
    bv.check()
    for g, r, mg in zip(grids, rhs, batch):
        alone = solver(g)
        alone.initialize(torch.zeros_like(r), r)
        p = alone.advance(3)
        assert torch.equal(p, mg.workspace.p[0])


@pytest.mark.parametrize('shapes', [[(256, 64)], [(32, 8), (64, 16), (16, 4)], [(512, 128), (8, 4), (384, 96)]])
def test_batched_vcycles_fp64_single_and_coarse_only_batches(shapes):
    """FP64 workspaces with FP64 coarsest solves; a batch of one; a batch
    whose instances all run wholly in one CTA (no launched level); a mix of
    two launched levels with a tiny instance."""
    from afsi_gpu_b200.batch import BatchedVCycles
    from afsi_gpu_b200.grid import ChannelGrid
    from afsi_gpu_b200.multigrid import ChannelMultigrid
    rng = np.random.default_rng(len(shapes))
    grids = [ChannelGrid(s, (4., 1.)) for s in shapes]

    def solver(g):
        return ChannelMultigrid(g, device=DEV, dtype=torch.float64, backend='b200')
    rhs = [torch.as_tensor(rng.standard_normal(s), device=DEV) for s in shapes]
    batch = [solver(g) for g in grids]
    bv = BatchedVCycles(batch, rhs)
    bv.run(3)
    again = [solver(g) for g in grids]
    pv = BatchedVCycles(again, rhs)
    pv.run(3, persistent=True)
    torch.cuda.synchronize()
    pv.check()
    for a, b in zip(batch, again):
        assert torch.equal(a.workspace.p[0], b.workspace.p[0])
    for g, r, mg in zip(grids, rhs, batch):
        alone = solver(g)
        alone.initialize(torch.zeros_like(r), r)
        assert torch.equal(alone.advance(3), mg.workspace.p[0])


def test_batched_vcycles_reject_what_they_do_not_batch():
    from afsi_gpu_b200.batch import BatchedVCycles
    from afsi_gpu_b200.grid import ChannelGrid
    from afsi_gpu_b200.multigrid import ChannelMultigrid
    g = ChannelGrid((64, 16), (4., 1.))
    a = ChannelMultigrid(g, device=DEV, dtype=torch.float32, coarse_dtype=torch.float64, backend='b200')
    b = ChannelMultigrid(g, device=DEV, dtype=torch.float64, backend='b200')
    rb = ChannelMultigrid(g, device=DEV, dtype=torch.float32, coarse_dtype=torch.float64, backend='b200',
                          smoother='red-black')
    for pair in ((a, b), (a, rb)):
        with pytest.raises(ValueError, match='batched V-cycles'):
            BatchedVCycles(list(pair))
    # a batch without right-hand-side sources starts from a zero iterate on
    # the right-hand side already in the workspace (the refinement's use)
    a.workspace.p[0].fill_(3.)
    a.workspace.rhs[0].copy_(torch.randn(g.shape, device=DEV))
    rhs = a.workspace.rhs[0].clone()
    BatchedVCycles([a]).run(1)
    alone = ChannelMultigrid(g, device=DEV, dtype=torch.float32, coarse_dtype=torch.float64, backend='b200')
    alone.initialize(torch.zeros_like(rhs), rhs)
    assert torch.equal(a.workspace.rhs[0], rhs) and torch.equal(a.workspace.p[0], alone.advance(1))


def test_refined_batch_meets_the_fp64_tolerance_per_instance_against_the_oracle():
    """The batching form at the FP64 bar: FP64 transfers and FP32 V-cycles in
    batched FP64 refinement.  Every instance meets its own FP64 tolerance
    (1e-10 relative residual), and every output is within 1e-8 (relative to
    its largest value) of the FP64 oracle: the transfers of
    ``mac2d/transfer.py:61-127`` and the channel solve of
    ``mac2d/multigrid.py:85-111`` run to 1e-10.  The device loop (one graph)
    equals the host-driven loop of the same kernels bit for bit."""
    from oracle import mg as oracle_mg
    b = seeded_batch(7, seed=5, shapes=((64, 16), (128, 32), (256, 64), (32, 8)), points=(800, 3000), device=DEV,
                     transfer_dtype=torch.float64,
                     schedule=Schedule(smoother='jacobi', cycles=4, vcycles='batched', refined=True))
    b.replay()
    torch.cuda.synchronize()
    b.check()
    rep = b.refined_report()
    assert rep['unconverged'] == 0 and not rep['nonfinite'] and rep['max_norm_over_tol'] <= 1
    assert all(c is not None and c > 0 for c in rep['cycles_to_tolerance'])
    graph_p = b.refinement().p.clone()
    for i, g in enumerate(b.grids):
        lo, hi = b.point_offsets[i], b.point_offsets[i + 1]
        ids, w = oracle.prepare2d(b.x[lo:hi].cpu().numpy(), g.shape, g.spacing)
        force = b.force[lo:hi].cpu().numpy()
        fields = b.fields(i)
        vel = (b.u_in[b.u_offsets[i]:b.u_offsets[i + 1]], b.v_in[b.v_offsets[i]:b.v_offsets[i + 1]])
        for c in range(2):
            ref = oracle.indexed_spread(force[:, c], ids[c], w[c], fields[c].numel(), g.volume)
            got = fields[c].reshape(-1).cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()
            ref = oracle.indexed_gather(vel[c].cpu().numpy(), ids[c], w[c])
            got = b.velocities(i)[:, c].cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()
        rhs = b.rhs64[i].cpu().numpy()
        pref, info = oracle_mg.solve(oracle_mg.Hierarchy(g.shape, g.spacing, 'channel'), rhs)
        p = b.pressure(i).cpu().numpy()
        assert np.abs(p - pref).max() <= 1e-8 * np.abs(pref).max(), i
        res = np.linalg.norm(rhs - oracle_mg.Hierarchy(g.shape, g.spacing, 'channel').apply(0, p))
        assert res <= 1e-10 * np.linalg.norm(rhs)
    st = b.refinement().run_launched(4)
    torch.cuda.synchronize()
    assert st['unconverged'] == 0
    assert torch.equal(b.refinement().p, graph_p)


def test_refined_batch_stops_at_the_refinement_cap_without_hanging():
    """A cap below what the tolerance needs ends the device loop with the
    instances reported unconverged (the loop cannot run past the cap)."""
    from afsi_gpu_b200.batch import BatchedRefinement
    b = seeded_batch(3, seed=6, shapes=((128, 32),), points=(500, 800), device=DEV, transfer_dtype=torch.float64)
    r = BatchedRefinement(b.solvers('jacobi'), b.rhs64, rtol=1e-14, atol=0., max_refinements=2)
    r.run(1)
    st = r.state()
    assert st['refinements'] == 2 and st['unconverged'] == 3
    assert all(d == -1 for d in st['done_at'])
