"""CN Helmholtz sweeps and Stokes residual reductions (csrc/stokes.cu) against
the reference's CPU kernel object and grid operators (B200).

Tolerances: Helmholtz fields bitwise in FP64 (the kernels keep the
reference's operation order without contraction); FP32 2e-6 of the field
scale. Reductions 1e-12 relative (block sums in another order; the blocked
momentum residual multiplies by 1/h^2 as the reference's blocked kernel does,
where its CPU branch divides by h^2).
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import stokes as ostokes
from afsi_gpu_b200.grid import MACGrid
from afsi_gpu_b200.helmholtz import (HelmholtzKernels, HelmholtzSolver, pressure_input_partial,
                                     pressure_norm_partial, residual_partial, start_partial)

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def _case(dtype=torch.float64):
    g = golden('stokes')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']))
    t = lambda a: torch.as_tensor(np.asarray(a), device=DEV, dtype=dtype)
    faces = lambda name: tuple(t(g[f'{name}{c}']) for c in range(3))
    return g, grid, t, faces


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_helmholtz_kernels_match_reference(dtype):
    g, grid, t, faces = _case(dtype)
    k = HelmholtzKernels()
    b, d = faces('b'), faces('d')
    params = t([g['alpha'], g['scale']])
    for tag, p in (('p', t(g['p'])), ('nop', None)):
        rhs = tuple(torch.empty_like(v) for v in b)
        cur = tuple(torch.empty_like(v) for v in b)
        nxt = tuple(torch.empty_like(v) for v in b)
        k.initialize(b, p, d, rhs, cur, params, grid)
        for c in range(3):
            for got, ref in ((rhs[c], g[f'{tag}_rhs{c}']), (cur[c], g[f'{tag}_init{c}'])):
                if dtype == torch.float64:
                    assert np.array_equal(got.cpu().numpy(), ref)
                else:
                    np.testing.assert_allclose(got.double().cpu().numpy(), ref, rtol=2e-6,
                                               atol=2e-6 * np.abs(ref).max())
        for _ in range(3):
            k.sweep(cur, rhs, d, nxt, params, grid)
            cur, nxt = nxt, cur
        for c in range(3):
            ref = g[f'{tag}_sweep3_{c}']
            if dtype == torch.float64:
                assert np.array_equal(cur[c].cpu().numpy(), ref)
            else:
                np.testing.assert_allclose(cur[c].double().cpu().numpy(), ref, rtol=2e-6,
                                           atol=2e-6 * np.abs(ref).max())


@pytest.mark.parametrize('graph', [True, False])
def test_helmholtz_solver_matches_reference(graph):
    """Initialize + 3 sweeps through the solver (one captured graph per
    pressure mode, or launched) equal the reference kernel object's chain."""
    g, grid, t, faces = _case()
    hs = HelmholtzSolver(grid, faces('d'), float(g['alpha']), 3, graph=graph)
    for _ in range(2):  # capture on the first solve, replay on the second
        u = hs.solve(faces('b'), t(g['p']), float(g['scale']))
        for c in range(3):
            assert np.array_equal(u[c].cpu().numpy(), g[f'p_sweep3_{c}'])
    u = hs.solve(faces('b'))
    for c in range(3):
        assert np.array_equal(u[c].cpu().numpy(), g[f'nop_sweep3_{c}'])
    # staged inputs and a caller-owned output
    for dst, src in zip(hs.inputs, faces('b')):
        dst.copy_(src)
    hs.pressure.copy_(t(g['p']))
    out = tuple(torch.empty_like(v) for v in u)
    hs.solve(pressure=True, pressure_scale=float(g['scale']), staged=True, out=out)
    for c in range(3):
        assert np.array_equal(out[c].cpu().numpy(), g[f'p_sweep3_{c}'])
    assert hs.calls == 4
    with pytest.raises(ValueError, match='sweep count'):
        HelmholtzSolver(grid, faces('d'), .1, 0)


def test_stokes_partials_reduce_to_reference_metrics():
    g, grid, t, faces = _case()
    n = int(np.prod(grid.shape))
    blocks = (n + 255) // 256
    p = t(g['p'])
    part = torch.empty((blocks, 3), device=DEV, dtype=torch.float64)
    start_partial(faces('b'), p, part, grid.shape)
    tot = part.sum(0)
    got = torch.stack((tot[0].sqrt(), tot[1] / n, (part[:, 2].amin() > 0).double())).cpu().numpy()
    np.testing.assert_allclose(got, g['start'], rtol=1e-12, atol=1e-15)
    alpha, scale = float(g['alpha']), float(g['scale'])
    coef = t([alpha, scale, 1 / scale, *(1 / h for h in grid.spacing), *(1 / (h * h) for h in grid.spacing)])
    residual = torch.empty(grid.shape, device=DEV, dtype=torch.float64)
    part2 = torch.empty((blocks, 2), device=DEV, dtype=torch.float64)
    residual_partial(faces('u'), p, faces('b'), residual, part2, grid.shape, coef)
    np.testing.assert_allclose(part2.sum(0).sqrt().cpu().numpy(), g['norms'], rtol=1e-12)
    np.testing.assert_allclose(residual.cpu().numpy(), g['residual'], rtol=1e-12,
                               atol=1e-12 * np.abs(g['residual']).max())
    rhs = t(g['prhs'])
    inputs = torch.empty((blocks, 5), device=DEV, dtype=torch.float64)
    pressure_input_partial(rhs, p, inputs)
    sums = inputs[:, :3].sum(0).cpu().numpy()
    np.testing.assert_allclose(sums, g['pmetrics'][:3], rtol=1e-12, atol=1e-12)
    assert inputs[:, 3:].amin().item() == 1
    norms = torch.empty((blocks, 2), device=DEV, dtype=torch.float64)
    pressure_norm_partial(rhs, p, norms, t([h * h for h in grid.spacing]))
    np.testing.assert_allclose(norms.sum(0).sqrt().cpu().numpy(), g['pmetrics'][3:], rtol=1e-12)
    bad = p.clone()
    bad[1, 2, 3] = float('inf')
    pressure_input_partial(rhs, bad, inputs)
    assert inputs[:, 4].amin().item() == 0 and inputs[:, 3].amin().item() == 1


def test_helmholtz_on_a_64_cube_against_the_oracle():
    """A larger grid (several blocks per face lattice) against the oracle."""
    grid = MACGrid((64, 48, 40), (1., .75, .625))
    rng = np.random.default_rng(2)
    b = ostokes.zero_normal([rng.standard_normal(grid.face_shape(c)) for c in range(3)])
    d = [1.5 + rng.random(grid.face_shape(c)) for c in range(3)]
    p = rng.standard_normal(grid.shape)
    rhs_ref, u_ref = ostokes.helmholtz_initialize(b, p, d, .3, grid.spacing)
    for _ in range(4):
        u_ref = ostokes.helmholtz_sweep(u_ref, rhs_ref, d, .02, grid.spacing)
    hs = HelmholtzSolver(grid, tuple(torch.as_tensor(x, device=DEV) for x in d), .02, 4)
    u = hs.solve(tuple(torch.as_tensor(x, device=DEV) for x in b), torch.as_tensor(p, device=DEV), .3)
    for c in range(3):
        assert np.array_equal(u[c].cpu().numpy(), u_ref[c])


# --------------------------------------------------------------- FGMRES solve

def _fgmres_case(precision='fp64'):
    from afsi_gpu_b200.stokes_fgmres import CNStokes
    z = golden('fgmres')
    grid = MACGrid(tuple(int(n) for n in z['shape']), tuple(float(x) for x in z['lengths']))
    flow = CNStokes(grid, dt=float(z['dt']), rho=float(z['rho']), mu=float(z['mu']), precision=precision)
    return z, grid, flow


def test_stokes_action_and_preconditioner_match_reference():
    """The packed action kernel equals the reference's action (bitwise up to
    the sign of zeros); the preconditioner (Helmholtz sweeps, the rhs kernel,
    the multigrid solve to 0.01, the result kernel) within 1e-12."""
    from afsi_gpu_b200.stokes_fgmres import _precondition
    from afsi_gpu_b200 import _lib
    z, grid, flow = _fgmres_case()
    v = flow.pack(tuple(torch.as_tensor(z[f'v{c}'], device=DEV) for c in range(3)), torch.as_tensor(z['q'], device=DEV))
    out = torch.empty_like(v)
    _lib.call('afsi_b200_stokes_action', v.data_ptr(), out.data_ptr(), flow._shape, flow._spacing, flow.alpha,
              min(grid.spacing), _lib.F64, _lib.stream())
    u, q = flow.unpack(out)
    for c in range(3):
        assert np.array_equal(u[c].cpu().numpy(), z[f'action_u{c}'])
    assert np.array_equal(q.cpu().numpy(), z['action_q'])
    pre, cycles = _precondition(flow, v, min(grid.spacing))
    u, q = flow.unpack(pre)
    assert cycles == int(z['pre_cycles'])
    for c in range(3):
        ref = z[f'pre_u{c}']
        np.testing.assert_allclose(u[c].cpu().numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_allclose(q.cpu().numpy(), z['pre_q'], rtol=0, atol=1e-12 * np.abs(z['pre_q']).max())


@pytest.mark.parametrize('tag', ['zero', 'warm'])
def test_fgmres_solve_matches_reference(tag):
    """The whole CN saddle-point solve against the reference's: identical
    iteration, action, Poisson-solve and V-cycle counts, velocity and pressure
    within 1e-10 of the reference's largest values, accepted by the same
    true-residual test."""
    z, grid, flow = _fgmres_case()
    b = tuple(torch.as_tensor(z[f'b{c}'], device=DEV) for c in range(3))
    initial = None if tag == 'zero' else torch.as_tensor(z['p0'], device=DEV)
    res = flow.stokes(b, initial)
    st, pr = res.diagnostics['stokes'], res.diagnostics['pressure']
    ref = z[f'{tag}_info']
    assert [st['iterations'], st['operator_actions'], pr['poisson_solves'], pr['cycles']] == [int(v) for v in ref[:4]]
    assert st['momentum_residual'] <= st['momentum_tolerance'] and st['divergence_norm'] <= st['divergence_tolerance']
    np.testing.assert_allclose(st['momentum_tolerance'], ref[5], rtol=1e-12)
    np.testing.assert_allclose(st['divergence_tolerance'], ref[7], rtol=1e-12)
    for c in range(3):
        r = z[f'{tag}_u{c}']
        np.testing.assert_allclose(res.velocity[c].cpu().numpy(), r, rtol=0, atol=1e-10 * np.abs(r).max())
    np.testing.assert_allclose(res.pressure.cpu().numpy(), z[f'{tag}_p'], rtol=0,
                               atol=1e-10 * np.abs(z[f'{tag}_p']).max())


def test_fgmres_precision_form_meets_the_fp64_acceptance_on_a_larger_grid():
    """FP32 preconditioner (Helmholtz sweeps and V-cycles; FP64 coarsest
    solve) inside the FP64 FGMRES: accepted by the FP64 true-residual test,
    and within 1e-8 of the FP64 oracle's solve on a 32^3 grid."""
    from afsi_gpu_b200.stokes_fgmres import CNStokes
    from oracle import mg as omg
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    rng = np.random.default_rng(31)
    b = [rng.standard_normal(grid.face_shape(c)) for c in range(3)]
    P = ostokes.StokesProblem(grid.shape, grid.spacing, 1e-3, 1., .01, omg.Hierarchy(grid.shape, grid.spacing,
                                                                                      'neumann'))
    u_ref, p_ref, info = ostokes.fgmres_solve(P, b)
    for precision in ('fp64', 'fp32-preconditioner'):
        flow = CNStokes(grid, dt=1e-3, rho=1., mu=.01, precision=precision)
        res = flow.stokes(tuple(torch.as_tensor(x, device=DEV) for x in b))
        st = res.diagnostics['stokes']
        assert st['momentum_residual'] <= st['momentum_tolerance']
        assert st['divergence_norm'] <= st['divergence_tolerance']
        if precision == 'fp64':
            assert st['iterations'] == info['iterations']
        for c in range(3):
            assert np.abs(res.velocity[c].cpu().numpy() - u_ref[c]).max() <= 1e-8 * np.abs(u_ref[c]).max()
        assert np.abs(res.pressure.cpu().numpy() - p_ref).max() <= 1e-8 * np.abs(p_ref).max()
