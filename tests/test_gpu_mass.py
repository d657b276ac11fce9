"""Consistent-mass Jacobi-PCG (csrc/mass.cu) against the reference MassSolver
solves and the oracle (B200).

The golden solves were made by the reference ``MassSolver``
(``mac/mass_solver.py:39-103``) on a P2 block mesh; the device solver must
take the same number of iterations and return the same solution.
Tolerances: FP64 solutions 1e-10 relative (the reductions are summed in
another order than torch's, so only rounding may differ; the solve itself
stops at rtol 1e-12); tolerances and residual norms 1e-12 relative; FP32
solutions 2e-4 relative at rtol 1e-5.
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import pcg as opcg
from afsi_gpu_b200 import _lib
from afsi_gpu_b200.mass import GraphMassSolver, MassSolver, SolverOptions

pytestmark = pytest.mark.gpu
DEV = 'cuda'
SCHEDULES = dict(default=dict(check_every=4), warm=dict(check_every=4), busy=dict(check_every=1, recompute_every=5))


def _options(**kw):
    return SolverOptions(rtol=kw.pop('rtol', 1e-12), atol=kw.pop('atol', 1e-13),
                         max_iterations=kw.pop('max_iterations', 500), **kw)


def _matrix(g, dtype=torch.float64):
    n = g['crow'].size - 1
    return torch.sparse_csr_tensor(torch.as_tensor(g['crow']), torch.as_tensor(g['col']),
                                   torch.as_tensor(g['values'], dtype=dtype), (n, n)).to(DEV)


def _spd(n, cols, seed, dtype=torch.float64, band=6):
    """Banded SPD matrix with a dominant positive diagonal (numpy CSR + torch)."""
    rng = np.random.default_rng(seed)
    rows, colsi, vals = [], [], []
    for i in range(n):
        for j in range(max(0, i - band), min(n, i + band + 1)):
            rows.append(i)
            colsi.append(j)
    rows, colsi = np.array(rows), np.array(colsi)
    lo = np.minimum(rows, colsi)
    hi = np.maximum(rows, colsi)
    sym = np.sin(lo * 1.7 + hi * 0.3 + seed) * 0.1  # symmetric off-diagonal values
    vals = np.where(rows == colsi, 2.0 + rng.random(n)[rows], sym)
    crow = np.zeros(n + 1, dtype=np.int64)
    np.add.at(crow, rows + 1, 1)
    crow = np.cumsum(crow)
    diag = vals[rows == colsi]
    M = torch.sparse_csr_tensor(torch.as_tensor(crow), torch.as_tensor(colsi), torch.as_tensor(vals, dtype=dtype),
                                (n, n)).to(DEV)
    rhs = rng.standard_normal((n, cols))
    return crow, colsi, vals, diag, rhs, M


@pytest.mark.parametrize('loop', ['graph', 'host'])
@pytest.mark.parametrize('name', list(SCHEDULES))
def test_golden_reference_solves(name, loop):
    g = golden('mass')
    M = _matrix(g)
    diagonal = torch.as_tensor(g['diagonal'], device=DEV)[:, None].expand(-1, 3)
    solver = MassSolver(M, diagonal, _options(**SCHEDULES[name]), loop=loop)
    rhs = torch.as_tensor(g['rhs'], device=DEV)
    initial = torch.as_tensor(g['initial'], device=DEV) if name == 'warm' else None
    x, info = solver.solve(rhs, initial)
    assert info.iterations == int(g[f'{name}_iterations'])
    assert info.residual_norm <= info.tolerance
    assert abs(info.tolerance - float(g[f'{name}_tolerance'])) <= 1e-12 * info.tolerance
    ref = g[f'{name}_x']
    np.testing.assert_allclose(x.cpu().numpy(), ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    # the solver is reusable: a second solve repeats the first exactly
    x2, info2 = solver.solve(rhs, initial)
    assert info2 == info and torch.equal(x2, x)


def test_graph_solver_matches_oracle_on_banded_system():
    crow, col, vals, diag, rhs, M = _spd(20000, 3, seed=3)
    opts = dict(check_every=4, recompute_every=40)
    x_ref, it_ref, res_ref, tol_ref = opcg.solve(crow, col, vals, diag, rhs, **opts)
    d = torch.as_tensor(diag, device=DEV)[:, None].expand(-1, 3)
    x, info = GraphMassSolver(M, d, _options(**opts)).solve(torch.as_tensor(rhs, device=DEV))
    assert abs(info.iterations - it_ref) <= 1
    assert info.residual_norm <= info.tolerance
    assert abs(info.tolerance - tol_ref) <= 1e-12 * tol_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-9, atol=1e-11 * np.abs(x_ref).max())


@pytest.mark.parametrize('cols', [1, 2])
def test_fp32_two_dimensional_blocks(cols):
    crow, col, vals, diag, rhs, M = _spd(3000, cols, seed=5, dtype=torch.float32)
    opts = dict(rtol=1e-5, atol=1e-7, check_every=2)
    x_ref, *_ = opcg.solve(crow, col, vals, diag, rhs, **opts)
    d = torch.as_tensor(diag, device=DEV, dtype=torch.float32)
    d = d if cols == 1 else d[:, None].expand(-1, cols)
    b = torch.as_tensor(rhs if cols > 1 else rhs[:, 0], device=DEV, dtype=torch.float32)
    x, info = MassSolver(M, d, _options(**opts)).solve(b)
    assert info.residual_norm <= info.tolerance
    np.testing.assert_allclose(x.cpu().numpy().reshape(x_ref.shape), x_ref, rtol=2e-4,
                               atol=2e-4 * np.abs(x_ref).max())


def test_zero_rhs_and_exact_initial_return_without_iterations():
    g = golden('mass')
    M = _matrix(g)
    diagonal = torch.as_tensor(g['diagonal'], device=DEV)[:, None].expand(-1, 3)
    solver = MassSolver(M, diagonal, _options(check_every=4))
    x, info = solver.solve(torch.zeros(diagonal.shape, device=DEV, dtype=torch.float64))
    assert info.iterations == 0 and info.residual_norm == 0 and info.tolerance == 1e-13
    assert not x.any()
    exact = torch.as_tensor(g['default_x'], device=DEV)
    _, info = solver.solve(M @ exact, exact)
    assert info.iterations == 0 and info.residual_norm <= info.tolerance


def test_not_converged_message_matches_oracle():
    g = golden('mass')
    M = _matrix(g)
    diagonal = torch.as_tensor(g['diagonal'], device=DEV)[:, None].expand(-1, 3)
    opts = dict(check_every=2, max_iterations=7)
    with pytest.raises(opcg.PCGError) as ref:
        opcg.solve(g['crow'], g['col'], g['values'], g['diagonal'], g['rhs'], **opts)
    for loop in ('graph', 'host'):
        with pytest.raises(RuntimeError) as got:
            MassSolver(M, diagonal, _options(**opts), loop=loop).solve(torch.as_tensor(g['rhs'], device=DEV))
        assert str(got.value).startswith('PCG did not converge: ')
        ref_norm = float(str(ref.value).split(': ')[1].split(' > ')[0])
        got_norm = float(str(got.value).split(': ')[1].split(' > ')[0])
        assert abs(got_norm - ref_norm) <= 1e-5 * ref_norm


def test_breakdown_on_indefinite_matrix_matches_oracle():
    # positive diagonal, indefinite matrix: [[1, 2], [2, 1]] blocks
    n = 64
    rows = np.repeat(np.arange(n), 2)
    col = np.stack([np.arange(n), np.arange(n) ^ 1], 1).reshape(-1)
    col = np.sort(col.reshape(n, 2), axis=1).reshape(-1)
    vals = np.where(rows == col, 1.0, 2.0)
    crow = np.arange(0, 2 * n + 1, 2, dtype=np.int64)
    diag = np.ones(n)
    rhs = np.zeros((n, 3))
    rhs[::2, 0] = 1.0
    rhs[1::2, 0] = -1.0
    with pytest.raises(opcg.PCGError, match='PCG breakdown'):
        opcg.solve(crow, col, vals, diag, rhs, check_every=1)
    M = torch.sparse_csr_tensor(torch.as_tensor(crow), torch.as_tensor(col), torch.as_tensor(vals),
                                (n, n)).to(DEV)
    d = torch.ones((n, 3), device=DEV, dtype=torch.float64)
    for loop in ('graph', 'host'):
        with pytest.raises(RuntimeError, match='PCG breakdown: operator/preconditioner must be positive definite'):
            MassSolver(M, d, _options(check_every=1), loop=loop).solve(torch.as_tensor(rhs, device=DEV))


def test_input_validation_messages():
    g = golden('mass')
    M = _matrix(g)
    diagonal = torch.as_tensor(g['diagonal'], device=DEV)[:, None].expand(-1, 3)
    solver = MassSolver(M, diagonal, _options())
    rhs = torch.as_tensor(g['rhs'], device=DEV)
    with pytest.raises(ValueError, match='mass solve shape, dtype or device mismatch'):
        solver.solve(rhs[:, :2])
    with pytest.raises(ValueError, match='mass solve shape, dtype or device mismatch'):
        solver.solve(rhs.float())
    bad = rhs.clone()
    bad[3, 1] = float('nan')
    with pytest.raises(ValueError, match='finite mass RHS and initial guess required'):
        solver.solve(bad)
    init = torch.zeros_like(rhs)
    init[0, 0] = float('inf')
    with pytest.raises(ValueError, match='finite mass RHS and initial guess required'):
        solver.solve(rhs, init)
    # a failed solve leaves the solver usable
    _, info = solver.solve(rhs)
    assert info.iterations > 0 and info.residual_norm <= info.tolerance
    neg = diagonal.clone()
    neg[5] = -1.0
    with pytest.raises(ValueError, match='Jacobi diagonal must be finite and positive'):
        MassSolver(M, neg)
    with pytest.raises(ValueError, match='graph PCG requires check_every in'):
        GraphMassSolver(M, diagonal, _options(check_every=17))


def test_solver_launches_native_kernels():
    g = golden('mass')
    M = _matrix(g)
    diagonal = torch.as_tensor(g['diagonal'], device=DEV)[:, None].expand(-1, 3)
    solver = MassSolver(M, diagonal, _options(check_every=4))
    before = _lib.launch_count()
    _, info = solver.solve(torch.as_tensor(g['rhs'], device=DEV))
    # begin + initial residual, then spmv/update/check per iteration
    assert _lib.launch_count() - before == 2 + 3 * info.iterations
