"""CUDA multigrid against the reference fixtures and the oracle (B200).

Tolerances follow the reference's own tests
(``tests/test_mac_multigrid_fused.py:13-86``, ``tests/test_valve_execution.py:13-41``):
level kernels 2e-12 (FP64) / 2e-5 (FP32), one V-cycle 2e-11, solves 2e-8.
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import mg as oracle
from afsi_gpu_b200 import synthetic
from afsi_gpu_b200.grid import MACGrid, ChannelGrid
from afsi_gpu_b200.multigrid import (B200Kernels, GeometricMultigrid, ChannelMultigrid, DirichletMultigrid,
                                     MGOptions, RefinedMultigrid)

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def t(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dtype)


def close(actual, expected, rtol, atol):
    np.testing.assert_allclose(actual.detach().cpu().double().numpy(), np.asarray(expected), rtol=rtol, atol=atol)


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_3d_level_kernels_match_reference_fixture(dtype):
    g = golden('mg3d')
    spacing = tuple(float(x) for x in g['spacing'])
    k = B200Kernels('neumann')
    pp, rr = t(g['pp'], dtype), t(g['rr'], dtype)
    out = torch.full_like(pp, float('nan'))
    tol = (0, 0) if dtype == torch.float64 else (2e-5, 2e-5)
    scale = float(np.abs(g['residual']).max())
    k.residual(pp, rr, out, spacing)
    close(out, g['residual'], tol[0], tol[1] * scale)
    k.smooth(pp, rr, None, out, spacing)
    close(out, g['smoothed'], tol[0], tol[1] * scale)
    coarse = torch.empty(tuple(n // 2 for n in g['pp'].shape), device=DEV, dtype=dtype)
    k.restrict(pp, coarse)
    close(coarse, g['restricted'], *tol)
    k.residual_restrict(pp, rr, coarse, spacing)
    close(coarse, g['residual_restricted'], tol[0], tol[1] * scale)
    k.restrict(pp, coarse)
    fine = pp.clone()
    k.prolong_add(coarse, fine)
    close(fine, g['prolonged'], 2e-15 if dtype == torch.float64 else 2e-5, 2e-15 if dtype == torch.float64 else 2e-5)
    const = torch.full_like(pp, 7.)
    k.residual(const, torch.zeros_like(pp), out, spacing)
    assert out.abs().max().item() == 0


def test_3d_single_block_cycle_and_solve_match_reference_fixture():
    g = golden('mg3d')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']))
    mg = GeometricMultigrid(grid, options=MGOptions(smooth=int(g['smooth'])), backend='b200')
    rhs, start = g['rhs'], g['start']
    mg.initialize(t(start), t(rhs - rhs.mean()))
    cyc = mg.cycle().clone()
    close(cyc, g['cycle'], 2e-11, 2e-12)
    p, info = mg.solve(t(rhs), t(start))
    assert info['cycles'] == int(g['cycles'])
    close(p, g['solution'], 2e-8, 2e-9)


@pytest.mark.parametrize('shape', [(32, 32, 32), (64, 64, 64), (16, 16, 32), (8, 12, 16)])
def test_3d_fused_cycle_matches_oracle(shape):
    grid = MACGrid(shape, tuple(n / 32 for n in shape))
    rng = np.random.default_rng(2)
    rhs = rng.standard_normal(shape)
    rhs -= rhs.mean()
    start = .1 * rng.standard_normal(shape)
    start -= start.mean()
    for smooth in (4, 3):
        h = oracle.Hierarchy(shape, grid.spacing, 'neumann')
        ref = oracle.cycle(h, 0, start, rhs, smooth)
        mg = GeometricMultigrid(grid, options=MGOptions(smooth=smooth), backend='b200')
        mg.initialize(t(start), t(rhs))
        got = mg.cycle()
        close(got, ref, 2e-11, 2e-11 * np.abs(ref).max())
        pm = GeometricMultigrid(grid, options=MGOptions(smooth=smooth), backend='b200-persistent')
        pm.initialize(t(start), t(rhs))
        close(pm.advance(1), ref, 2e-11, 2e-11 * np.abs(ref).max())
        # two cycles in one launch equal two single launches
        pm.initialize(t(start), t(rhs))
        two = pm.advance(2).clone()
        mg.initialize(t(start), t(rhs))
        mg.cycle()
        close(two, mg.cycle().cpu().numpy(), 1e-13, 1e-13 * np.abs(ref).max())


def test_3d_solve_matches_reference_fixture_and_oracle_and_graphs():
    g = golden('mg3d')
    shape2 = tuple(int(n) for n in g['shape2'])
    grid = MACGrid(shape2, tuple(float(x) for x in g['lengths2']))
    for backend in ('b200', 'b200-graph', 'b200-persistent'):
        mg = GeometricMultigrid(grid, backend=backend)
        p, info = mg.solve(t(g['rhs2']))
        assert info['cycles'] == int(g['cycles2'])
        close(p, g['solution2'], 2e-8, 2e-9)
        assert info['residual_norm'] <= info['tolerance']
    grid = MACGrid((64, 64, 64), (1., 1., 1.))
    rhs = synthetic.mean_free_normal(grid.shape, seed=9).numpy()
    ref, rinfo = oracle.solve(oracle.Hierarchy(grid.shape, grid.spacing, 'neumann'), rhs)
    for backend in ('b200-graph', 'b200-persistent'):
        mg = GeometricMultigrid(grid, backend=backend)
        p, info = mg.solve(t(rhs))
        assert info['cycles'] == rinfo['cycles']
        close(p, ref, 2e-8, 2e-9 * np.abs(ref).max())


def test_3d_solver_contract_errors_buffers_and_ownership():
    grid = MACGrid((16, 16, 16), (1., 1., 1.))
    mg = GeometricMultigrid(grid, backend='b200-graph')
    rhs = t(synthetic.mean_free_normal(grid.shape, seed=1).numpy())
    before = [x.data_ptr() for x in (*mg.workspace.p, *mg.workspace.ping, *mg.workspace.rhs)]
    rhs_copy = rhs.clone()
    p, _ = mg.solve(rhs)
    p_copy = p.clone()
    p2, _ = mg.solve(-rhs, p)
    close(p2, (-p_copy).cpu().numpy(), 1e-7, 1e-8)
    assert torch.equal(p, p_copy) and torch.equal(rhs, rhs_copy)
    assert before == [x.data_ptr() for x in (*mg.workspace.p, *mg.workspace.ping, *mg.workspace.rhs)]
    zero, info = mg.solve(torch.zeros_like(rhs))
    assert info['cycles'] == 0 and zero.count_nonzero().item() == 0
    with pytest.raises(ValueError, match='incompatible'):
        mg.solve(torch.ones_like(rhs))
    with pytest.raises(ValueError, match='invalid pressure RHS'):
        mg.solve(torch.full_like(rhs, float('nan')))
    with pytest.raises(ValueError, match='CUDA'):
        GeometricMultigrid(grid, device='cpu')


def test_channel_kernels_cycle_solve_match_reference_fixture():
    g = golden('mg2d')
    grid = ChannelGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']))
    k = B200Kernels('channel')
    pp, rhs = t(g['pp']), t(g['rhs'])
    out = torch.empty_like(pp)
    k.residual(pp, rhs, out, grid.spacing)
    close(out, g['residual'], 0, 0)
    k.smooth(pp, rhs, None, out, grid.spacing)
    close(out, g['smoothed'], 0, 0)
    coarse = torch.empty(tuple(n // 2 for n in grid.shape), device=DEV, dtype=torch.float64)
    k.residual_restrict(pp, rhs, coarse, grid.spacing)
    close(coarse, g['residual_restricted'], 0, 0)
    fine = pp.clone()
    k.prolong_add(coarse, fine)
    close(fine, g['prolonged'], 1e-14, 1e-13)
    mg = ChannelMultigrid(grid, backend='b200')
    mg.initialize(t(g['start']), rhs)
    close(mg.cycle(), g['cycle'], 2e-12, 2e-13)
    p, info = mg.solve(rhs)
    assert info['cycles'] == int(g['cycles'])
    close(p, g['solution'], 2e-8, 2e-9)
    big = ChannelGrid(tuple(int(n) for n in g['shape_b']), tuple(float(x) for x in g['lengths_b']))
    for backend in ('b200', 'b200-graph', 'b200-persistent'):
        mg = ChannelMultigrid(big, backend=backend)
        p, info = mg.solve(t(g['rhs_b']))
        assert info['cycles'] == int(g['cycles_b'])
        close(p, g['solution_b'], 2e-8, 2e-9 * np.abs(g['solution_b']).max())


@pytest.mark.parametrize('bc', ['channel', 'periodic'])
def test_2d_fused_cycle_matches_oracle(bc):
    shape = (256, 64)
    grid = ChannelGrid(shape, (1., .25), periodic=bc == 'periodic')
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal(shape)
    if bc == 'periodic':
        rhs -= rhs.mean()
    start = .1 * rng.standard_normal(shape)
    h = oracle.Hierarchy(shape, grid.spacing, bc)
    if bc == 'periodic':
        start -= start.mean()
    ref = oracle.cycle(h, 0, start, rhs, 4)
    mg = ChannelMultigrid(grid, backend='b200')
    mg.initialize(t(start), t(rhs))
    close(mg.cycle(), ref, 2e-11, 2e-11 * np.abs(ref).max())
    pref, rinfo = oracle.solve(h, rhs)
    for backend in ('b200-graph', 'b200-persistent'):
        p, info = ChannelMultigrid(grid, backend=backend).solve(t(rhs))
        assert info['cycles'] == rinfo['cycles']
        close(p, pref, 2e-8, 2e-9 * np.abs(pref).max())
    mg = ChannelMultigrid(grid, backend='b200-persistent')
    mg.initialize(t(start), t(rhs))
    close(mg.advance(1), ref, 2e-11, 2e-11 * np.abs(ref).max())


def test_fp32_multigrid_converges_with_fp64_coarse_solve():
    grid = MACGrid((64, 64, 64), (1., 1., 1.))
    rhs = synthetic.mean_free_normal(grid.shape, seed=2)
    mg = GeometricMultigrid(grid, dtype=torch.float32, coarse_dtype=torch.float64,
                            options=MGOptions(rtol=1e-5), backend='b200-graph')
    p, info = mg.solve(rhs.to(DEV, torch.float32))
    ref, _ = oracle.solve(oracle.Hierarchy(grid.shape, grid.spacing, 'neumann'), rhs.numpy())
    err = np.abs(p.double().cpu().numpy() - ref).max() / np.abs(ref).max()
    assert info['residual_norm'] <= info['tolerance'] and err < 1e-4


def test_device_solve_loop_follows_the_host_check_schedule():
    """The graph backend's device-side loop (WHILE graph node) runs the same
    cycles as the host loop: blocks of check_every with a residual check after
    each, the tail past the last full block on the host; results bitwise equal."""
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    rhs = synthetic.mean_free_normal(grid.shape, seed=6).to(DEV)
    hopeless = MGOptions(max_cycles=5, check_every=2, rtol=1e-300, atol=1e-300)
    host = GeometricMultigrid(grid, options=hopeless, backend='b200')
    dev = GeometricMultigrid(grid, options=hopeless, backend='b200-graph')
    assert dev.loop_graph
    for mg in (host, dev):
        with pytest.raises(RuntimeError, match='did not converge'):
            mg.solve(rhs)
    assert torch.equal(host.workspace.p[0], dev.workspace.p[0])  # 5 cycles each
    for check_every in (1, 3):
        opts = MGOptions(check_every=check_every)
        a, ia = GeometricMultigrid(grid, options=opts, backend='b200').solve(rhs)
        b, ib = GeometricMultigrid(grid, options=opts, backend='b200-graph').solve(rhs)
        assert ia['cycles'] == ib['cycles'] and ia['cycles'] % check_every == 0
        assert torch.equal(a, b) and ia['residual_norm'] == ib['residual_norm']
    cgrid = ChannelGrid((64, 16), (4., 1.))
    crhs = torch.as_tensor(np.random.default_rng(3).standard_normal(cgrid.shape), device=DEV)
    a, ia = ChannelMultigrid(cgrid, backend='b200').solve(crhs)
    b, ib = ChannelMultigrid(cgrid, backend='b200-graph').solve(crhs)
    assert ia['cycles'] == ib['cycles'] and torch.equal(a, b)


def test_dirichlet_multigrid_matches_reference_fixture_and_oracle():
    """Open box, zero face pressure (reference ``mac/dirichlet_mg.py``;
    ``tests/test_paper_lv.py:74-86``): solves with the reference's cycle count,
    the manufactured field to 1e-8, one V-cycle 2e-11, level kernels 2e-12."""
    g = golden('dirichlet')
    shape = tuple(int(n) for n in g['shape'])
    grid = MACGrid(shape, tuple(float(x) for x in g['lengths']))
    for backend in ('b200', 'b200-graph', 'b200-persistent', 'graph'):
        solver = DirichletMultigrid(grid, backend=backend)
        p, info = solver.solve(t(g['rhs']))
        assert info['cycles'] == int(g['cycles'])
        close(p, g['solution'], 2e-8, 2e-9)
        close(p, g['exact'], 1e-8, 1e-8)
        assert info['residual_norm'] <= info['tolerance']
        saved = p.clone()
        zero, zinfo = solver.solve(torch.zeros_like(p))
        assert zinfo['cycles'] == 0 and torch.equal(zero, torch.zeros_like(p))
        assert torch.equal(p, saved)  # returned solutions are owned copies
    mg = DirichletMultigrid(grid, backend='b200')
    mg.initialize(t(g['p']), t(g['r']))
    close(mg.cycle(), g['cycle'], 2e-11, 2e-11 * np.abs(g['cycle']).max())
    k = B200Kernels('dirichlet')
    spacing = grid.spacing
    out = torch.empty(shape, device=DEV, dtype=torch.float64)
    k.residual(t(g['p']), t(g['r']), out, spacing)
    close(out, g['r'] - g['apply'], 2e-12, 2e-12 * np.abs(g['apply']).max())
    fine = torch.zeros(shape, device=DEV, dtype=torch.float64)
    k.prolong_add(t(g['coarse']), fine)
    close(fine, g['prolonged'], 1e-14, 1e-14)
    h = oracle.Hierarchy(shape, spacing, 'dirichlet')
    d = torch.empty(shape, device=DEV, dtype=torch.float64)
    k.smooth(t(g['p']), t(g['r']), t(h.diagonals[0]), d, spacing)
    ref = g['p'] + (2 / 3) * (g['r'] - g['apply']) / h.diagonals[0]
    close(d, ref, 2e-12, 2e-12 * np.abs(ref).max())
    shape2 = tuple(int(n) for n in g['shape2'])
    grid2 = MACGrid(shape2, tuple(float(x) for x in g['lengths2']))
    pref, rinfo = oracle.solve(oracle.Hierarchy(shape2, grid2.spacing, 'dirichlet'), g['rhs2'])
    for backend in ('b200-graph', 'b200-persistent'):
        p2, info2 = DirichletMultigrid(grid2, backend=backend).solve(t(g['rhs2']))
        assert info2['cycles'] == rinfo['cycles'] == int(g['cycles2'])
        close(p2, g['solution2'], 2e-8, 2e-9 * np.abs(g['solution2']).max())
    with pytest.raises(ValueError, match='nonfinite Dirichlet pressure input'):
        bad = t(g['rhs']).clone()
        bad[0, 0, 0] = float('nan')
        solver.solve(bad)
    with pytest.raises(ValueError, match='shape/dtype/device mismatch'):
        solver.solve(t(g['rhs']).float())


def _fp64_residual(solver_cls, grid, p, rhs, **kw):
    """||rhs - A p|| by the FP64 solver's own residual kernel."""
    mg = solver_cls(grid, backend='b200', **kw)
    mg.initialize(p, rhs)
    return mg.residual_norm().item()


@pytest.mark.parametrize('case', ['neumann64', 'channel', 'periodic', 'dirichlet'])
def test_refined_fp32_multigrid_reaches_fp64_tolerance(case):
    """Precision form: FP32 V-cycles inside FP64 iterative refinement meet the
    FP64 solver's tolerance (1e-10 relative) measured in FP64, and the
    solution agrees with the FP64 oracle at the solve tolerance (2e-8, the
    solve bar of the reference's tests)."""
    if case == 'neumann64':
        grid, bc, cls = MACGrid((64, 64, 64), (1., 1., 1.)), 'neumann', GeometricMultigrid
        rhs = synthetic.mean_free_normal(grid.shape, seed=8).numpy()
    elif case == 'dirichlet':
        grid, bc, cls = MACGrid((32, 32, 32), (1., 1., 1.)), 'dirichlet', DirichletMultigrid
        rhs = np.random.default_rng(9).standard_normal(grid.shape)
    else:
        grid = ChannelGrid((256, 64), (1., .25), periodic=case == 'periodic')
        bc, cls = case, ChannelMultigrid
        rhs = np.random.default_rng(10).standard_normal(grid.shape)
        if case == 'periodic':
            rhs -= rhs.mean()
    refined = RefinedMultigrid(grid, bc=bc)
    p, info = refined.solve(t(rhs))
    assert p.dtype == torch.float64
    assert info['refinements'] >= 1 and info['residual_norm'] <= info['tolerance']
    rhs_shifted = rhs - rhs.mean() if bc in ('neumann', 'periodic') else rhs
    assert abs(info['tolerance'] - max(1e-12, 1e-10 * np.linalg.norm(rhs_shifted))) <= 1e-12 * info['tolerance']
    assert _fp64_residual(cls, grid, p, t(rhs_shifted)) <= info['tolerance'] * (1 + 1e-6)
    pref, _ = oracle.solve(oracle.Hierarchy(grid.shape, grid.spacing, bc), rhs)
    close(p, pref, 2e-8, 2e-8 * np.abs(pref).max())
    if bc in ('neumann', 'periodic'):
        assert abs(p.mean().item()) <= 1e-14 * p.abs().max().item()
    # a second solve with the first as the initial guess needs no refinement
    _, again = refined.solve(t(rhs), p)
    assert again['refinements'] == 0


def test_refined_multigrid_rejects_bad_input():
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    refined = RefinedMultigrid(grid)
    rhs = synthetic.mean_free_normal(grid.shape, seed=1).to(DEV)
    with pytest.raises(ValueError, match='FP64'):
        refined.solve(rhs.float())
    with pytest.raises(ValueError, match='incompatible Neumann'):
        refined.solve(rhs + 1.0)
    bad = rhs.clone()
    bad[0, 0, 0] = float('nan')
    with pytest.raises(ValueError, match='finite'):
        refined.solve(bad)
    p, info = refined.solve(rhs)
    assert info['residual_norm'] <= info['tolerance']


@pytest.mark.parametrize('case', ['neumann', 'channel', 'periodic', 'dirichlet'])
def test_red_black_smoother_matches_oracle(case):
    """Selectable red-black Gauss-Seidel smoother (a method change; the
    reference has only weighted Jacobi): one V-cycle equals the oracle's
    red-black cycle to 2e-11 (the V-cycle bar), solves take the oracle's cycle
    count and agree with it to 2e-8, and with the Jacobi solve at the solve
    tolerance (2e-8 of the field)."""
    if case in ('neumann', 'dirichlet'):
        grid = MACGrid((32, 32, 32), (1., 1., 1.))
        cls = GeometricMultigrid if case == 'neumann' else DirichletMultigrid
    else:
        grid = ChannelGrid((256, 64), (1., .25), periodic=case == 'periodic')
        cls = ChannelMultigrid
    rng = np.random.default_rng(12)
    rhs = rng.standard_normal(grid.shape)
    start = .1 * rng.standard_normal(grid.shape)
    if case in ('neumann', 'periodic'):
        rhs -= rhs.mean()
        start -= start.mean()
    h = oracle.Hierarchy(grid.shape, grid.spacing, case)
    opts = MGOptions(smooth=2)
    ref = oracle.cycle(h, 0, start, rhs, 2, 'red-black')
    mg = cls(grid, backend='b200', smoother='red-black', options=opts)
    mg.initialize(t(start), t(rhs))
    close(mg.cycle(), ref, 2e-11, 2e-11 * np.abs(ref).max())
    pref, rinfo = oracle.solve(h, rhs, sweeps=2, smoother='red-black')
    pjac, _ = oracle.solve(h, rhs)
    for backend in ('b200', 'b200-graph'):
        p, info = cls(grid, backend=backend, smoother='red-black', options=opts).solve(t(rhs))
        assert info['cycles'] == rinfo['cycles'] and info['backend'].endswith('red-black')
        assert info['residual_norm'] <= info['tolerance']
        close(p, pref, 2e-8, 2e-9 * np.abs(pref).max())
        close(p, pjac, 2e-8, 2e-8 * np.abs(pjac).max())


def test_red_black_smoother_option_checks():
    grid = MACGrid((16, 16, 16), (1., 1., 1.))
    with pytest.raises(ValueError, match='smoother'):
        GeometricMultigrid(grid, smoother='sor')
    with pytest.raises(ValueError, match='Jacobi smoother only'):
        GeometricMultigrid(grid, smoother='red-black', backend='b200-persistent')
    refined = RefinedMultigrid(grid, smoother='red-black', options=MGOptions(smooth=2))
    rhs = synthetic.mean_free_normal(grid.shape, seed=3).to(DEV)
    p, info = refined.solve(rhs)
    assert info['residual_norm'] <= info['tolerance'] and info['backend'].endswith('red-black-refined')


def test_deferred_solves_equal_synchronous_solves():
    """solve_deferred queues the started loop graph and reads later: two
    solves queued back to back give, read in either order, the solutions,
    cycle counts and norms of the synchronous solves; bad input raises at
    result() as solve raises it."""
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    mg = GeometricMultigrid(grid)
    rhs = [synthetic.mean_free_normal(grid.shape, seed=s).to(DEV) for s in (21, 22)]
    sync = [mg.solve(r) for r in rhs]
    pending = [mg.solve_deferred(r) for r in rhs]
    for (p, info), pend in zip(reversed(sync), reversed(pending)):
        q, qinfo = pend.result()
        assert torch.equal(p, q)
        assert qinfo['cycles'] == info['cycles'] and qinfo['residual_norm'] == info['residual_norm']
        assert pend.result()[0] is q  # read once
    bad = rhs[0] + 1.0  # net flux
    pend = mg.solve_deferred(bad)
    with pytest.raises(ValueError, match='incompatible'):
        pend.result()
    # a deferred solve whose device loop leaves host cycles, read after a later solve
    short = GeometricMultigrid(grid, options=MGOptions(max_cycles=5))
    first = short.solve_deferred(rhs[0], rtol=1e-30)
    later = short.solve_deferred(rhs[1])
    with pytest.raises(RuntimeError, match='did not converge'):
        first.result()
    with pytest.raises(RuntimeError, match='did not converge'):
        later.result()
