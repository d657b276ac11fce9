"""Table-free element transfers (csrc/fe_fused.cu) on the B200.

P2 without stencil tables and the matrix-free P1 element transfer (the
reference's ``AdaptiveP1Transfer`` CUDA execution, ``mac/adaptive_cell.py:
22-83``): each point's position, bases and weights formed inside the
transfer kernel.  Tolerances: 1e-12 of the field scale against the reference
fixtures and the FP64 oracle (the single-instance parity bar); 1e-14 against
the table-based kernels on the same rule (same arithmetic, another order of
atomic additions); 3e-6 for FP32 transfers beside FP64 positions against the
FP64 oracle.
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import ib as oracle, csr as ocsr
from afsi_gpu_b200 import synthetic, p2_cuda_transfer as p2t
from afsi_gpu_b200.grid import MACGrid
from afsi_gpu_b200.quadrature import InteractionRule, QuadratureGroup

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def t(a, dtype=None):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dtype)


def close(got, ref, tol):
    ref = np.asarray(ref)
    got = got.double().cpu().numpy().reshape(ref.shape) if torch.is_tensor(got) else np.asarray(got)
    assert np.abs(got - ref).max() <= tol * max(np.abs(ref).max(), 1e-300), np.abs(got - ref).max()


def _free(x, rule):
    return p2t.TableFreeStencil(x, rule, torch.zeros((), dtype=torch.int32, device=DEV))


def test_p2_table_free_matches_reference_fixture_and_table_kernels():
    g = golden('p2')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))
    groups = tuple(QuadratureGroup(t(g[f'cells{k}']), t(g[f'N{k}']), t(g[f'W{k}']), int(g[f'order{k}']))
                   for k in range(int(g['ngroups'])))
    rule = InteractionRule(groups, None, sum(gr.weights.numel() for gr in groups))
    x = t(g['x'])
    tr = p2t.P2Transfer(grid, t(g['X']), t(g['cells0']))
    st = _free(x, rule)
    fields = p2t.spread(tr, t(g['coef']), st)
    vel = tuple(t(g[f'v{c}']) for c in range(3))
    rhs = p2t.assemble_velocity(tr, vel, st)
    tr.check(st)
    base, phi = p2t.prepare(tr, x, rule)
    tab = p2t.SharedAdaptiveStencil(base, phi, rule)
    tf, tr_rhs = p2t.spread(tr, t(g['coef']), tab), p2t.assemble_velocity(tr, vel, tab)
    for c in range(3):
        close(fields[c], g[f'u{c}'], 1e-12)
        close(fields[c], tf[c].cpu().numpy(), 1e-14)
    close(rhs, g['rhs'], 1e-12)
    close(rhs, tr_rhs.cpu().numpy(), 1e-14)


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_p2_table_free_shell_against_oracle(dtype):
    """A multi-group rule on a 64^3 grid: FP64 within 1e-12 of the oracle;
    FP32 transfers beside FP64 positions within 3e-6 of the FP64 oracle; the
    deferred table-free prepare confirms its rule."""
    X, cells = synthetic.p2_shell(2, 12, 16, inner=(.125, .075, .075), outer=(.16, .11, .11))
    grid = MACGrid((64, 64, 64), (1., 1., 1.))
    Xd = t(X)
    tr = p2t.P2Transfer(grid, Xd, t(cells), max_order=22, transfer_dtype=dtype)
    deferred = tr.prepare_table_free(Xd)
    st = tr.confirm(deferred)
    deferred = tr.prepare_table_free(Xd)  # second call: the cached rule, no host read until confirm
    st2 = deferred.stencil
    assert st2.rule is st.rule and len(st.rule.groups) > 1
    rng = np.random.default_rng(8)
    coef = rng.standard_normal((X.shape[0], 3))
    vel = synthetic.fourier_velocity3d(grid, seed=1)
    fields = tr.spread(t(coef, dtype), st2)
    rhs = tr.assemble_velocity(tuple(v.to(DEV, dtype) for v in vel), st2)
    assert tr.confirm(deferred) is st2
    full = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in st.rule.groups]
    ob, op, invalid = oracle.p2_prepare(X, [(c, N) for c, N, _ in full], grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    tol = 1e-12 if dtype == torch.float64 else 3e-6
    ref = oracle.p2_spread(coef, full, ob, op, grid.shape, grid.volume)
    for c in range(3):
        close(fields[c], ref[c], tol)
    ref = oracle.p2_gather_assemble([v.numpy() for v in vel], full, ob, op, grid.shape, X.shape[0])
    close(rhs, ref, tol)


@pytest.mark.parametrize('name', ['pair', 'block'])
def test_p1_matrix_free_transfer_matches_reference_operators(name):
    """The matrix-free P1 transfer against the reference's assembled operators
    (``AssembledP1Transfer``, fixture p1csr): spread = B^T coef / volume,
    interpolate = B u, on the reference's own rule."""
    g = golden('p1csr')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))
    X = t(g[f'{name}_X'])
    groups = tuple(QuadratureGroup(t(g[f'{name}_cells{k}']), t(g[f'{name}_N{k}']), t(g[f'{name}_W{k}']),
                                   int(g[f'{name}_N{k}'].shape[0])) for k in range(int(g[f'{name}_ngroups'])))
    rule = InteractionRule(groups, None, sum(gr.weights.numel() for gr in groups))
    tr = p2t.P1Transfer(grid, X, t(g[f'{name}_cells']))
    st = _free(X, rule)
    rng = np.random.default_rng(4)
    coef = rng.standard_normal((X.shape[0], 3))
    vel = [rng.standard_normal(grid.face_shape(c)) for c in range(3)]
    fields = tr.spread(t(coef), st)
    rhs = tr.interpolate_rhs(tuple(t(v) for v in vel), st)
    tr.check(st)
    for c in range(3):
        crow, col, val = g[f'{name}_crow{c}'], g[f'{name}_col{c}'], g[f'{name}_val{c}']
        nf = int(np.prod(grid.face_shape(c)))
        tcrow, tcol, tval = ocsr.csr_transpose(crow, col, val, nf)
        close(fields[c].reshape(-1), ocsr.csr_matvec(tcrow, tcol, tval, coef[:, c]) / grid.volume, 1e-12)
        close(rhs[:, c], ocsr.csr_matvec(crow, col, val, vel[c].reshape(-1)), 1e-12)


def test_p1_transfer_adaptive_rule_chunks_and_precision_form():
    """P1Transfer's own adaptive rule (orders as the reference's ``_orders``),
    with a point density that gives rules of more than 64 points (the kernels'
    chunked path), against the oracle; FP32 transfers within 3e-6."""
    X, cells = synthetic.prolate_shell(2, 10, 16, inner=(.125, .075, .075), outer=(.16, .11, .11))
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    Xd = t(X)
    tr = p2t.P1Transfer(grid, Xd, t(cells), point_density=6., max_order=12)
    st = tr.prepare(Xd)
    assert max(gr.values.shape[0] for gr in st.rule.groups) > 64
    np.testing.assert_array_equal(st.rule.orders.cpu().numpy(),
                                  oracle.p1_orders(X, cells, min(grid.spacing), 6.))
    full = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in st.rule.groups]
    ob, op, invalid = oracle.p2_prepare(X, [(c, N) for c, N, _ in full], grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    rng = np.random.default_rng(9)
    coef = rng.uniform(-1, 1, (X.shape[0], 3))
    vel = synthetic.fourier_velocity3d(grid, seed=2)
    ref_f = oracle.p2_spread(coef, full, ob, op, grid.shape, grid.volume)
    ref_r = oracle.p2_gather_assemble([v.numpy() for v in vel], full, ob, op, grid.shape, X.shape[0])
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 3e-6)):
        tr = p2t.P1Transfer(grid, Xd, t(cells), point_density=6., max_order=12, transfer_dtype=dtype)
        st = tr.prepare(Xd)
        fields = tr.spread(t(coef, dtype), st)
        rhs = tr.interpolate_rhs(tuple(v.to(DEV, dtype) for v in vel), st)
        tr.check(st)
        for c in range(3):
            close(fields[c], ref_f[c], tol)
        close(rhs, ref_r, tol)


def test_table_free_support_and_connectivity_errors_do_not_trap():
    """A point whose support leaves the grid, and a node id out of range, are
    flagged by the transfer kernels (skipped, no trap) and raised by check."""
    X, cells = synthetic.prolate_shell(1, 6, 8, inner=(.125, .075, .075), outer=(.16, .11, .11))
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    Xd = t(X)
    tr = p2t.P1Transfer(grid, Xd, t(cells))
    st = tr.prepare(Xd)
    moved = Xd.clone()
    moved[torch.as_tensor(cells[0], device=DEV)] = torch.tensor([.01, .5, .5], device=DEV, dtype=torch.float64)
    bad = p2t.TableFreeStencil(moved, st.rule, torch.zeros((), dtype=torch.int32, device=DEV))
    fields = tr.spread(t(np.ones((X.shape[0], 3))), bad)
    assert all(torch.isfinite(f).all() for f in fields)
    with pytest.raises(ValueError, match='support'):
        tr.check(bad)
    broken = st.rule.groups[0].cells.clone()
    broken[0, 1] = X.shape[0] + 5
    groups = (QuadratureGroup(broken, st.rule.groups[0].values, st.rule.groups[0].weights, 0),) + st.rule.groups[1:]
    rule = InteractionRule(groups, None, st.rule.point_count)
    bad = p2t.TableFreeStencil(Xd, rule, torch.zeros((), dtype=torch.int32, device=DEV))
    tr.assemble_velocity(tuple(v.to(DEV) for v in synthetic.fourier_velocity3d(grid, seed=3)), bad)
    with pytest.raises(RuntimeError, match='connectivity'):
        tr.check(bad)


def test_deferred_flags_are_read_from_the_pinned_copy():
    """note_transfers copies a table-free stencil's flag word behind its
    transfers; confirm then raises the support flag from that copy."""
    X, cells = synthetic.prolate_shell(1, 6, 8, inner=(.125, .075, .075), outer=(.16, .11, .11))
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    Xd = t(X)
    tr = p2t.P1Transfer(grid, Xd, t(cells))
    tr.confirm(tr.prepare_table_free(Xd))
    ok = tr.prepare_table_free(Xd)
    tr.spread(t(np.ones((X.shape[0], 3))), ok.stencil)
    tr.note_transfers(ok)
    assert tr.confirm(ok) is ok.stencil
    moved = Xd - torch.tensor([.45, 0., 0.], device=DEV, dtype=torch.float64)  # the same rule, part outside
    bad = tr.prepare_table_free(moved)
    tr.spread(t(np.ones((X.shape[0], 3))), bad.stencil)
    tr.note_transfers(bad)
    with pytest.raises(ValueError, match='support'):
        tr.confirm(bad)


@pytest.mark.parametrize('kind', ['p2', 'p1', 'p2-fp32'])
def test_deterministic_table_free_transfers_are_reproducible(kind):
    """The deterministic table-free forms use no atomics.  The spread writes
    each element's box to a scratch slot and reduces the boxes per 4x4x4 face
    tile in a fixed order.  The gather-assemble writes element sums and
    reduces them per node.  Two runs are bitwise equal.  They match the
    atomic table-free forms within 1e-14 of the scale and the FP64 oracle
    within 1e-12.  P2 uses rules of several orders; P1 uses rules of more
    than 64 points, so the kernels' chunked path runs too.  The FP32
    transfers beside FP64 positions match their atomic form and the FP64
    oracle within 3e-6."""
    dtype = torch.float32 if kind == 'p2-fp32' else torch.float64
    if kind.startswith('p2'):
        X, cells = synthetic.p2_shell(2, 12, 16, inner=(.125, .075, .075), outer=(.16, .11, .11))
        grid = MACGrid((64, 64, 64), (1., 1., 1.))
        cls, kw = p2t.P2Transfer, dict(max_order=22, transfer_dtype=dtype)
    else:
        X, cells = synthetic.prolate_shell(2, 10, 16, inner=(.125, .075, .075), outer=(.16, .11, .11))
        grid = MACGrid((32, 32, 32), (1., 1., 1.))
        cls, kw = p2t.P1Transfer, dict(point_density=6., max_order=12)
    Xd = t(X)
    det = cls(grid, Xd, t(cells), deterministic=True, **kw)
    atomic = cls(grid, Xd, t(cells), **kw)
    st = det.confirm(det.prepare_table_free(Xd))
    assert isinstance(st, p2t.TableFreeStencil) and len(st.rule.groups) > 1
    rng = np.random.default_rng(21)
    coef = t(rng.standard_normal((X.shape[0], 3)), dtype)
    vel = tuple(v.to(DEV, dtype) for v in synthetic.fourier_velocity3d(grid, seed=5))
    f1, f2 = det.spread(coef, st), det.spread(coef, st)
    r1, r2 = det.assemble_velocity(vel, st), det.assemble_velocity(vel, st)
    det.check(st)
    fa, ra = atomic.spread(coef, st), atomic.assemble_velocity(vel, st)
    atomic.check(st)
    full = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in st.rule.groups]
    ob, op, invalid = oracle.p2_prepare(X, [(c, N) for c, N, _ in full], grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    ref_f = oracle.p2_spread(coef.double().cpu().numpy(), full, ob, op, grid.shape, grid.volume)
    ref_r = oracle.p2_gather_assemble([v.double().cpu().numpy() for v in vel], full, ob, op, grid.shape, X.shape[0])
    near, tol = (1e-14, 1e-12) if dtype == torch.float64 else (3e-6, 3e-6)
    for c in range(3):
        assert torch.equal(f1[c], f2[c])
        close(f1[c], fa[c].cpu().numpy(), near)
        close(f1[c], ref_f[c], tol)
    assert torch.equal(r1, r2)
    close(r1, ra.cpu().numpy(), near)
    close(r1, ref_r, tol)


def test_deterministic_spread_reports_boxes_beyond_its_slots():
    """Elements of a coarse shell on a 128^3 grid span more than 8 faces per
    axis, beyond the deterministic spread's slots: they set the overflow
    flag (no trap, finite fields) and check raises."""
    X, cells = synthetic.p2_shell(1, 6, 8, inner=(.125, .075, .075), outer=(.16, .11, .11))
    grid = MACGrid((128, 128, 128), (1., 1., 1.))
    Xd = t(X)
    det = p2t.P2Transfer(grid, Xd, t(cells), deterministic=True, max_order=26)
    st = det.confirm(det.prepare_table_free(Xd))
    fields = det.spread(t(np.ones((X.shape[0], 3))), st)
    assert all(torch.isfinite(f).all() for f in fields)
    with pytest.raises(RuntimeError, match='deterministic'):
        det.check(st)
