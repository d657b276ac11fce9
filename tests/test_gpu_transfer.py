"""CUDA IB transfers against the oracle and the reference fixtures (B200).

Tolerances: integer tables (bases, stencil ids) bit-exact; FP64 weights within
rounding of the reference torch path (its CPU sqrt is not correctly rounded);
FP64 spread/gather 1e-12 relative (the FP64 parity bar); FP32 8e-5/3e-5
(``tests/test_p2_cuda_execution.py:38`` of the reference).
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import ib as oracle
from afsi_gpu_b200 import _lib, cuda_ib, p2_cuda_transfer as p2t, synthetic
from afsi_gpu_b200.grid import MACGrid, ChannelGrid
from afsi_gpu_b200.quadrature import InteractionRule, QuadratureGroup

pytestmark = pytest.mark.gpu
DEV = 'cuda'
F64 = dict(rtol=1e-12, atol=1e-12)
F32 = dict(rtol=8e-5, atol=3e-5)


def t(a, dtype=None):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dtype)


def close(actual, expected, **tol):
    np.testing.assert_allclose(actual.detach().cpu().numpy() if torch.is_tensor(actual) else actual,
                               expected, **tol)


def scaled_tol(expected, rtol):
    """Relative bar on the field scale (values near cancellation get the field's scale)."""
    return dict(rtol=rtol, atol=rtol * float(np.abs(expected).max()))


# ----------------------------------------------------------------- compact 3D

def test_compact_prepare_matches_reference_fixture_and_oracle():
    g = golden('compact3d')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))
    pts = t(g['points'])
    st = cuda_ib.compact_prepare(grid, pts)
    assert torch.equal(st.base.cpu(), torch.as_tensor(g['base']))
    close(st.phi, g['phi'], rtol=0, atol=6e-17)
    sh = cuda_ib.compact_prepare(grid, pts, layout='shared')
    assert torch.equal(sh.base.cpu(), torch.as_tensor(g['shared_base']))
    close(sh.phi, g['shared_phi'], rtol=0, atol=6e-17)
    # the oracle restates the same IEEE arithmetic: bitwise equal
    ob, op = oracle.compact_prepare(g['points'], oracle.face_origins(grid.origin, grid.spacing), grid.spacing)
    assert np.array_equal(st.base.cpu().numpy(), ob) and np.array_equal(st.phi.cpu().numpy(), op)
    rad = cuda_ib.compact_prepare(grid, pts, layout='shared', phi_form='radical')
    rb, rp = oracle.compact_prepare(g['points'], oracle.shared_origins(grid.origin, grid.spacing), grid.spacing,
                                    form='radical')
    assert np.array_equal(rad.base.cpu().numpy(), rb) and np.array_equal(rad.phi.cpu().numpy(), rp)


def test_compact_spread_gather_match_reference_fixture():
    g = golden('compact3d')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))
    st = cuda_ib.compact_prepare(grid, t(g['points']))
    fields = cuda_ib.compact_spread(grid, t(g['force']), st)
    for c in range(3):
        close(fields[c], g[f'u{c}'], **scaled_tol(g[f'u{c}'], 1e-12))
    got = cuda_ib.compact_gather(grid, tuple(t(g[f'v{c}']) for c in range(3)), st)
    close(got, g['gathered'], **scaled_tol(g['gathered'], 1e-12))
    cuda_ib.check()


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_compact_transfer_large_random_against_oracle(dtype):
    rng = np.random.default_rng(1)
    grid = MACGrid((48, 40, 56), (1.2, 1., 1.4), (-.1, .2, .3))
    h = np.array(grid.spacing)
    lo = np.array(grid.origin) + 2.01 * h
    hi = np.array(grid.origin) + (np.array(grid.shape) - 2.01) * h
    pts = (lo + (hi - lo) * rng.random((200000, 3))).astype(np.float64)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    st = cuda_ib.compact_prepare(grid, t(pts.astype(npdt)))
    ob, op = oracle.compact_prepare(pts.astype(npdt), oracle.face_origins(grid.origin, grid.spacing, npdt),
                                    grid.spacing)
    if dtype == torch.float64:
        assert np.array_equal(st.base.cpu().numpy(), ob) and np.array_equal(st.phi.cpu().numpy(), op)
    force = rng.standard_normal((200000, 3)).astype(npdt)
    fields = cuda_ib.compact_spread(grid, t(force), st)
    ref = oracle.spread3d(force.astype(np.float64), ob, op.astype(np.float64), grid.shape, grid.volume)
    tol = 1e-12 if dtype == torch.float64 else 3e-5
    for c in range(3):
        close(fields[c].reshape(-1).double(), ref[c], **scaled_tol(ref[c], tol))
    vel = [rng.standard_normal(grid.face_shape(c)).astype(npdt) for c in range(3)]
    got = cuda_ib.compact_gather(grid, tuple(t(v) for v in vel), st)
    ref = oracle.gather3d([v.astype(np.float64) for v in vel], ob, op.astype(np.float64), grid.shape)
    close(got.double(), ref, **scaled_tol(ref, tol))
    cuda_ib.check()


def test_compact_support_and_index_errors_do_not_trap():
    grid = MACGrid((16, 16, 16), (1., 1., 1.))
    with pytest.raises(ValueError, match='support'):
        cuda_ib.compact_prepare(grid, t([[.01, .5, .5]]))
    pts = t([[.5, .5, .5]])
    st = cuda_ib.compact_prepare(grid, pts)
    bad = cuda_ib.CompactStencil(st.base.clone(), st.phi)
    bad.base[0, 0, 0] = 1000  # would address outside the grid
    fields = cuda_ib.compact_spread(grid, t([[1., 1., 1.]]), bad)
    with pytest.raises(RuntimeError, match='outside'):
        cuda_ib.check()
    assert fields[0].abs().sum().item() == 0  # the bad point was skipped
    assert fields[1].abs().sum().item() > 0


def test_spread_is_the_adjoint_of_gather():
    rng = np.random.default_rng(4)
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    pts = t(.2 + .6 * rng.random((5000, 3)))
    st = cuda_ib.compact_prepare(grid, pts)
    F = t(rng.standard_normal((5000, 3)))
    u = tuple(t(rng.standard_normal(grid.face_shape(c))) for c in range(3))
    fields = cuda_ib.compact_spread(grid, F, st)
    lhs = (F * cuda_ib.compact_gather(grid, u, st)).sum()
    rhs = grid.volume * sum((a * b).sum() for a, b in zip(u, fields))
    assert abs(lhs.item() - rhs.item()) <= 1e-12 * abs(lhs.item())


# ---------------------------------------------------------------------- 2D

def test_2d_prepare_and_indexed_transfer_match_reference_fixture():
    g = golden('transfer2d')
    grid = ChannelGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']))
    st = cuda_ib.prepare2d(grid, t(g['points']))
    for c in range(2):
        assert torch.equal(st.indices[c].cpu(), torch.as_tensor(g[f'ids{c}']))
        close(st.weights[c], g[f'w{c}'], rtol=0, atol=6e-17)
    ob, ow = oracle.prepare2d(g['points'], grid.shape, grid.spacing)
    for c in range(2):
        assert np.array_equal(st.weights[c].cpu().numpy(), ow[c])
    s = cuda_ib.spread2d(grid, t(g['force']), st)
    for c in range(2):
        close(s[c].reshape(-1), g[f's{c}'], **scaled_tol(g[f's{c}'], 1e-12))
    got = cuda_ib.gather2d((t(g['v0']), t(g['v1'])), st)
    close(got, g['gathered'], **scaled_tol(g['gathered'], 1e-12))
    with pytest.raises(ValueError, match='support'):
        cuda_ib.prepare2d(grid, t([[.01, .5]]))


def test_2d_config_ellipse_against_oracle():
    grid = ChannelGrid((256, 64), (1., .25), periodic=True)
    pts = synthetic.ellipse_points(20000, spacing=1 / 256, seed=3)
    st = cuda_ib.prepare2d(grid, t(pts))
    ob, ow = oracle.prepare2d(pts, grid.shape, grid.spacing)
    for c in range(2):
        assert np.array_equal(st.indices[c].cpu().numpy(), ob[c])
        assert np.array_equal(st.weights[c].cpu().numpy(), ow[c])
    force = np.random.default_rng(5).standard_normal((20000, 2))
    s = cuda_ib.spread2d(grid, t(force), st)
    vel = synthetic.fourier_velocity2d(grid, seed=2)
    got = cuda_ib.gather2d(tuple(v.to(DEV) for v in vel), st)
    for c in range(2):
        ref = oracle.indexed_spread(force[:, c], ob[c], ow[c], s[c].numel(), grid.volume)
        close(s[c].reshape(-1), ref, **scaled_tol(ref, 1e-12))
        ref = oracle.indexed_gather(vel[c].numpy(), ob[c], ow[c])
        close(got[:, c], ref, **scaled_tol(ref, 1e-12))


def test_raw_indexed_ops_general_neighbors_and_components():
    rng = np.random.default_rng(6)
    field = t(rng.standard_normal((500, 3)))
    ids = t(rng.integers(0, 500, (300, 64)))
    w = t(rng.standard_normal((300, 64)))
    got = cuda_ib.indexed_gather(field, ids, w)
    ref = (field[ids] * w[..., None]).sum(1)
    close(got, ref.cpu().numpy(), rtol=1e-12, atol=1e-12)
    f = t(rng.standard_normal((300, 3)))
    s = cuda_ib.indexed_spread(f, ids, w, 500, 2.)
    ref = torch.zeros(500, 3, device=DEV, dtype=torch.float64).index_add_(
        0, ids.reshape(-1), (w[..., None] * f[:, None, :] / 2.).reshape(-1, 3))
    close(s, ref.cpu().numpy(), rtol=1e-12, atol=1e-12)
    with pytest.raises(RuntimeError, match='shape mismatch'):
        cuda_ib.indexed_gather(field, ids, w[:, :3])


# ---------------------------------------------------------------------- P2

def _golden_p2():
    g = golden('p2')
    grid = MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))
    groups = tuple(QuadratureGroup(t(g[f'cells{k}']), t(g[f'N{k}']), t(g[f'W{k}']), int(g[f'order{k}']))
                   for k in range(int(g['ngroups'])))
    rule = InteractionRule(groups, None, sum(gr.weights.numel() for gr in groups))
    return g, grid, rule


def test_p2_raw_operators_match_reference_fixture():
    g, grid, rule = _golden_p2()
    X = t(g['X'])
    tr = p2t.P2Transfer(grid, X, t(g['cells0']))
    base, phi = p2t.prepare(tr, t(g['x']), rule)
    st = p2t.SharedAdaptiveStencil(base, phi, rule)
    eb, ep = st.expanded()
    assert torch.equal(eb.cpu(), torch.as_tensor(g['base']))
    close(ep, g['phi'], rtol=4e-12, atol=2e-15)
    fields = p2t.spread(tr, t(g['coef']), st)
    for c in range(3):
        close(fields[c], g[f'u{c}'], **scaled_tol(g[f'u{c}'], 1e-12))
    vel = tuple(t(g[f'v{c}']) for c in range(3))
    rhs = p2t.assemble_velocity(tr, vel, st)
    close(rhs, g['rhs'], **scaled_tol(g['rhs'], 1e-12))
    det = p2t.assemble_velocity_deterministic(tr, vel, st)
    close(det, g['rhs'], **scaled_tol(g['rhs'], 1e-12))
    # power identity coef·rhs = vol Σ u·f (reference test_p2_cuda_execution.py:53-55)
    solid = (t(g['coef']) * p2t.assemble_velocity(tr, vel, st)).sum()
    fluid = grid.volume * sum((u * f).sum() for u, f in zip(vel, fields))
    assert abs(solid.item() - fluid.item()) <= 1e-11 * abs(solid.item())
    cuda_ib.check()


SMALL = dict(inner=(.125, .075, .075), outer=(.16, .11, .11))


@pytest.mark.parametrize('dtype,n', [(torch.float64, 32), (torch.float32, 32), (torch.float64, 64)])
def test_p2_shell_against_oracle(dtype, n):
    """Half-size synthetic shell: 40k points in 2 quadrature groups on 32^3,
    324k points in 5 groups on 64^3.  Prepare bit-exact (FP64), spread and
    gather-assemble within the parity bar."""
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((n, n, n), (1., 1., 1.))
    npdt = np.float64 if dtype == torch.float64 else np.float32
    Xd = t(X.astype(npdt))
    tr = p2t.P2Transfer(grid, Xd, t(cells), max_order=22)
    st = tr.prepare(Xd)
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy().astype(npdt)) for gr in st.rule.groups]
    ob, op, invalid = oracle.p2_prepare(X.astype(npdt), groups, grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    if dtype == torch.float64:
        assert np.array_equal(st.base.cpu().numpy(), ob)
        assert np.array_equal(st.phi.cpu().numpy(), op)
    else:
        # FP32 knots may bin to the adjacent cell; the weights then differ, not the operator
        assert (st.base.cpu().numpy() != ob).mean() < 1e-4
    rng = np.random.default_rng(8)
    coef = rng.standard_normal((X.shape[0], 3))
    full = [(gr.cells.cpu().numpy(), gr.values.cpu().double().numpy(), gr.weights.cpu().double().numpy())
            for gr in st.rule.groups]
    b64, p64 = st.base.cpu().numpy(), st.phi.cpu().double().numpy()
    fields = tr.spread(t(coef.astype(npdt)), st)
    ref = oracle.p2_spread(coef, full, b64, p64, grid.shape, grid.volume)
    tol = 1e-12 if dtype == torch.float64 else 3e-5
    for c in range(3):
        close(fields[c].reshape(-1).double(), ref[c], **scaled_tol(ref[c], tol))
    vel = synthetic.fourier_velocity3d(grid, seed=1)
    rhs = tr.assemble_velocity(tuple(v.to(DEV, dtype) for v in vel), st)
    ref = oracle.p2_gather_assemble([v.numpy() for v in vel], full, b64, p64, grid.shape, X.shape[0])
    close(rhs.double(), ref, **scaled_tol(ref, tol))
    cuda_ib.check()


def test_p2_precision_form_fp32_transfers_with_fp64_positions():
    """Precision form: FP64 positions and bases (bit-exact with the FP64
    oracle), weights the FP64 weights rounded once to FP32, FP32 spread and
    gather-assemble within 3e-6 of the field scale of the FP64 oracle."""
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((64, 64, 64), (1., 1., 1.))
    tr = p2t.P2Transfer(grid, t(X), t(cells), max_order=22, transfer_dtype=torch.float32)
    st = tr.prepare(t(X))
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy()) for gr in st.rule.groups]
    ob, op, invalid = oracle.p2_prepare(X, groups, grid.origin, grid.spacing, grid.shape)
    assert invalid == 0 and st.phi.dtype == torch.float32
    assert np.array_equal(st.base.cpu().numpy(), ob)
    assert np.array_equal(st.phi.cpu().numpy(), op.astype(np.float32))
    st2 = tr.prepare(t(X))  # the speculative (rule reused) path keeps the precision form
    assert st2.phi.dtype == torch.float32 and torch.equal(st2.phi, st.phi)
    full = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in st.rule.groups]
    coef = np.random.default_rng(8).standard_normal((X.shape[0], 3))
    fields = tr.spread(t(coef, torch.float32), st)
    ref = oracle.p2_spread(coef, full, ob, op, grid.shape, grid.volume)
    for c in range(3):
        assert fields[c].dtype == torch.float32
        close(fields[c].reshape(-1).double(), ref[c], **scaled_tol(ref[c], 3e-6))
    vel = synthetic.fourier_velocity3d(grid, seed=1)
    rhs = tr.assemble_velocity(tuple(v.to(DEV, torch.float32) for v in vel), st)
    ref = oracle.p2_gather_assemble([v.numpy() for v in vel], full, ob, op, grid.shape, X.shape[0])
    close(rhs.double(), ref, **scaled_tol(ref, 3e-6))
    with pytest.raises(ValueError, match='dtype must match'):
        tr.spread(t(coef), st)


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_p2_deterministic_spread_is_reproducible_and_matches(dtype):
    """Tile-sorted, atomic-free spread: bitwise equal over repeated runs,
    equal to the atomic spread and to the FP64 oracle within the parity bar
    (1e-12 FP64; 3e-6 for FP32 transfers beside FP64 positions)."""
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((64, 64, 64), (1., 1., 1.))
    kw = dict(max_order=22, transfer_dtype=dtype)
    det = p2t.P2Transfer(grid, t(X), t(cells), deterministic=True, **kw)
    atomic = p2t.P2Transfer(grid, t(X), t(cells), **kw)
    st = det.prepare(t(X))
    coef = np.random.default_rng(11).standard_normal((X.shape[0], 3))
    c = t(coef, dtype)
    first = det.spread(c, st)
    second = det.spread(c, st)
    reference = atomic.spread(c, st)
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in st.rule.groups]
    ob, op, _ = oracle.p2_prepare(X, [(g[0], g[1]) for g in groups], grid.origin, grid.spacing, grid.shape)
    ref = oracle.p2_spread(coef, groups, ob, op, grid.shape, grid.volume)
    tol = 1e-12 if dtype == torch.float64 else 3e-6
    for k in range(3):
        assert torch.equal(first[k], second[k])
        close(first[k].double(), reference[k].double().cpu().numpy(), **scaled_tol(reference[k].double().cpu().numpy(), tol))
        close(first[k].reshape(-1).double(), ref[k], **scaled_tol(ref[k], tol))


def test_p2_deterministic_assembly_is_bitwise_reproducible():
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    tr = p2t.P2Transfer(grid, t(X), t(cells), deterministic=True, max_order=22)
    st = tr.prepare(t(X))
    vel = tuple(v.to(DEV) for v in synthetic.fourier_velocity3d(grid, seed=4))
    a = tr.assemble_velocity(vel, st)
    b = tr.assemble_velocity(vel, st)
    assert torch.equal(a, b)
    c = p2t.assemble_velocity(tr, vel, st)
    close(a, c.cpu().numpy(), **scaled_tol(c.cpu().numpy(), 1e-13))


def test_p2_support_violation_raises_value_error():
    X, cells = synthetic.p2_shell(1, 8, 12, **SMALL)
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    tr = p2t.P2Transfer(grid, t(X), t(cells), max_order=22)
    with pytest.raises(ValueError, match='support'):
        tr.prepare(t(X) - .45)


# ------------------------------------------------------------ adaptive orders

def _orders(x, cells, dx, density, last=None, bins=64):
    orders = torch.empty(cells.shape[0], dtype=torch.int64, device=DEV)
    summary = torch.full((3 + bins,), -7, dtype=torch.int32, device=DEV)
    _lib.call('afsi_b200_p2_orders', x.data_ptr(), x.shape[0], cells.data_ptr(), cells.shape[0], dx, density, 3,
              orders.data_ptr(), None if last is None else last.data_ptr(), summary.data_ptr(), bins,
              _lib.dtype_code(x.dtype), _lib.stream(x.device))
    return orders, summary.cpu().tolist()


def test_p2_orders_match_reference_fixture_and_count_changes():
    g = golden('orders')
    x, cells = t(g['x']), t(g['cells'])
    for k, (dx, density) in enumerate(zip(g['dx'], g['density'])):
        expected = g[f'p2_{k}']
        np.testing.assert_array_equal(oracle.p2_orders(g['x'], g['cells'], dx, density), expected)
        orders, summary = _orders(x, cells, float(dx), float(density))
        np.testing.assert_array_equal(orders.cpu().numpy(), expected)
        assert summary[0] == len(expected) and summary[1] == expected.max() and summary[2] == 0
        hist = np.bincount(expected, minlength=64)[:64]
        assert summary[3:] == hist.tolist()
        again, summary = _orders(x, cells, float(dx), float(density), last=orders)
        assert torch.equal(again, orders) and summary[0] == 0
        moved = orders.clone()
        moved[[3, 17, 400]] += 1
        _, summary = _orders(x, cells, float(dx), float(density), last=moved)
        assert summary[0] == 3
    # orders at or above the bin count are left out of the histogram, not the maximum
    orders, summary = _orders(x, cells, .011, 2., bins=8)
    top = int(g['p2_0'].max())
    assert summary[1] == top and sum(summary[3:]) == int((g['p2_0'] < 8).sum())


def test_p2_orders_flag_bad_connectivity_and_nonfinite_nodes():
    g = golden('orders')
    x, cells = t(g['x']), t(g['cells'])
    bad = cells.clone()
    bad[5, 7] = x.shape[0]
    orders, summary = _orders(x, bad, .011, 2.)
    assert summary[2] == _lib.FLAG_INDEX and orders[5].item() == 0
    assert orders[6].item() == int(g['p2_0'][6])
    xn = x.clone()
    xn[int(g['cells'][9, 0]), 1] = float('nan')
    orders, summary = _orders(xn, cells, .011, 2.)
    assert summary[2] == _lib.FLAG_SUPPORT and orders[9].item() == 0


def test_p2_deferred_prepare_confirms_the_rule_after_the_fact():
    """prepare_deferred reads nothing on the host: unchanged orders give the
    speculative tables bitwise equal to a synchronous prepare and confirm
    returns them as they are; changed orders make confirm prepare again with
    the new rule (equal to a synchronous prepare); a support violation is
    raised at confirm."""
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    tr = p2t.P2Transfer(grid, t(X), t(cells), max_order=22)
    ref = p2t.P2Transfer(grid, t(X), t(cells), max_order=22)
    first = tr.prepare_deferred(t(X))  # no cached rule yet: synchronous
    assert tr.confirm(first) is first.stencil
    second = tr.prepare_deferred(t(X))
    sync = ref.prepare(t(X))
    assert torch.equal(second.stencil.base, sync.base) and torch.equal(second.stencil.phi, sync.phi)
    assert tr.confirm(second) is second.stencil
    centre = X.mean(0)
    Y = centre + 1.3 * (X - centre)  # larger elements: higher orders
    third = tr.prepare_deferred(t(Y))
    assert third.stencil.rule is second.stencil.rule  # speculative, with the old rule
    fixed = tr.confirm(third)
    assert fixed.rule is not second.stencil.rule
    again = ref.prepare(t(Y))
    assert fixed.rule.point_count == again.rule.point_count
    assert torch.equal(fixed.base, again.base) and torch.equal(fixed.phi, again.phi)
    bad = tr.prepare_deferred(t(Y) - .45)  # a translation keeps the orders
    with pytest.raises(ValueError, match='support'):
        tr.confirm(bad)


def test_p2_transfer_prepare_reuses_the_rule_and_rebuilds_on_change():
    X, cells = synthetic.p2_shell(2, 12, 16, **SMALL)
    grid = MACGrid((32, 32, 32), (1., 1., 1.))
    tr = p2t.P2Transfer(grid, t(X), t(cells), max_order=22)
    first = tr.prepare(t(X))
    second = tr.prepare(t(X))  # speculative prepare with the cached rule
    assert second.rule is first.rule
    assert torch.equal(first.base, second.base) and torch.equal(first.phi, second.phi)
    centre = X.mean(0)
    Y = centre + 1.3 * (X - centre)  # larger elements: higher orders
    third = tr.prepare(t(Y))
    assert third.rule is not first.rule
    orders = oracle.p2_orders(Y, cells, min(grid.spacing), 2.)
    np.testing.assert_array_equal(third.rule.orders.cpu().numpy(), orders)
    assert third.rule.point_count == sum(len(gr.weights[0]) * gr.cells.shape[0] for gr in third.rule.groups)
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy()) for gr in third.rule.groups]
    ob, op, invalid = oracle.p2_prepare(Y, groups, grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    assert np.array_equal(third.base.cpu().numpy(), ob) and np.array_equal(third.phi.cpu().numpy(), op)
    # a translation keeps the orders: the speculative prepare reports the wall
    with pytest.raises(ValueError, match='support'):
        tr.prepare(t(Y) - .45)
