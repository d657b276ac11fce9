"""P1 CSR contraction, table-to-CSR and SpMV responses against the reference
operators and the oracle (B200).

Tolerances: CSR structure (row pointers, column indices) exact; values
3e-13 relative (FP64) — the reference itself sums a site's points in a
parallel tree and its table values atomically, so only rounding may differ
(``tests/test_csr_hash_assembly.py:210-212`` of the reference uses 3e-13);
FP32 3e-6 relative.  Responses 1e-12 relative on the field scale.
"""
import numpy as np
import pytest
import torch
from conftest import golden
from oracle import csr as ocsr, ib as oib
from afsi_gpu_b200 import _lib, cuda_ib
from afsi_gpu_b200.grid import MACGrid
from afsi_gpu_b200.p1_csr import HashWorkspace, MissingStream, P1CSRTransfer, power_of_two
from afsi_gpu_b200.p2_cuda_transfer import SharedAdaptiveStencil
from afsi_gpu_b200.quadrature import InteractionRule, QuadratureGroup

pytestmark = pytest.mark.gpu
DEV = 'cuda'


def t(a, dtype=None):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dtype)


def _grid(g):
    return MACGrid(tuple(int(n) for n in g['shape']), tuple(float(x) for x in g['lengths']),
                   tuple(float(x) for x in g['origin']))


def _golden_rule(g, name, dtype=torch.float64):
    groups = []
    for k in range(int(g[f'{name}_ngroups'])):
        groups.append(QuadratureGroup(t(g[f'{name}_cells{k}']), t(g[f'{name}_N{k}'], dtype),
                                      t(g[f'{name}_W{k}'], dtype), int(g[f'{name}_N{k}'].shape[0])))
    total = sum(gr.weights.numel() for gr in groups)
    return InteractionRule(tuple(groups), None, total)


def _tables(tr, x, rule):
    """Shared tables of a fixed rule through the P1 prepare kernel."""
    base = torch.empty((2, rule.point_count, 3), device=DEV, dtype=torch.int64)
    phi = x.new_empty((2, rule.point_count, 3, 4))
    word = _lib.status_word(x.device)
    word.zero_()
    g, offset = tr.grid, 0
    for gr in rule.groups:
        _lib.call('afsi_b200_p1_prepare', x.data_ptr(), x.shape[0], gr.cells.data_ptr(), gr.cells.shape[0],
                  gr.values.data_ptr(), gr.values.shape[0], _lib.doubles(g.origin), _lib.doubles(g.spacing),
                  _lib.doubles([n - 2 for n in g.shape]), base.data_ptr(), phi.data_ptr(), rule.point_count, offset,
                  word.data_ptr(), _lib.dtype_code(x.dtype), _lib.stream(x.device))
        offset += gr.weights.numel()
    assert int(word.item()) == 0
    return SharedAdaptiveStencil(base, phi, rule)


@pytest.mark.parametrize('name', ['pair', 'block'])
def test_p1_contraction_and_csr_match_reference_operators(name):
    g = golden('p1csr')
    grid = _grid(g)
    X = t(g[f'{name}_X'])
    tr = P1CSRTransfer(grid, X, t(g[f'{name}_cells']))
    rule = _golden_rule(g, name)
    st = _tables(tr, X, rule)
    groups = [(g[f'{name}_cells{k}'], g[f'{name}_N{k}']) for k in range(len(rule.groups))]
    ob, op, invalid = oib.p2_prepare(g[f'{name}_X'], groups, grid.origin, grid.spacing, grid.shape)
    assert invalid == 0
    assert np.array_equal(st.base.cpu().numpy(), ob) and np.array_equal(st.phi.cpu().numpy(), op)
    A = tr.assemble_stencil(st)
    for c in range(3):
        B, BT = A.gather[c], A.spread[c]
        assert np.array_equal(B.crow.cpu().numpy(), g[f'{name}_crow{c}'])
        assert np.array_equal(B.col.cpu().numpy(), g[f'{name}_col{c}'])
        np.testing.assert_allclose(B.val.cpu().numpy(), g[f'{name}_val{c}'], rtol=3e-13, atol=3e-16)
        tcrow, tcol, tval = ocsr.csr_transpose(g[f'{name}_crow{c}'], g[f'{name}_col{c}'], g[f'{name}_val{c}'],
                                               BT.shape[0])
        assert np.array_equal(BT.crow.cpu().numpy(), tcrow) and np.array_equal(BT.col.cpu().numpy(), tcol)
        np.testing.assert_allclose(BT.val.cpu().numpy(), tval, rtol=3e-13, atol=3e-16)
    assert A.assembly['total_nnz'] == sum(len(g[f'{name}_col{c}']) for c in range(3))


def test_p1_transfer_pipeline_rule_tables_and_responses_against_oracle():
    g = golden('p1csr')
    grid = _grid(g)
    Xn = g['block_X']
    cells = g['block_cells']
    tr = P1CSRTransfer(grid, t(Xn), t(cells))
    A = tr.prepare(t(Xn))
    orders = oib.p1_orders(Xn, cells, min(grid.spacing), 2.)
    np.testing.assert_array_equal(A.rule.orders.cpu().numpy(), orders)
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in A.rule.groups]
    base, phi, invalid = oib.p2_prepare(Xn, [(c, N) for c, N, _ in groups], grid.origin, grid.spacing, grid.shape)
    rng = np.random.default_rng(4)
    coef = rng.standard_normal((Xn.shape[0], 3))
    fields = tr.spread(t(coef), A)
    vel = [rng.standard_normal(grid.face_shape(c)) for c in range(3)]
    rhs = tr.interpolate_rhs(tuple(t(v) for v in vel), A)
    power_solid = 0.
    for c in range(3):
        fs = grid.face_shape(c)
        _, _, (crow, col, val) = ocsr.assemble(base, phi, groups, c, fs, Xn.shape[0])
        np.testing.assert_allclose(A.gather[c].val.cpu().numpy(), val, rtol=3e-13, atol=3e-16)
        tcrow, tcol, tval = ocsr.csr_transpose(crow, col, val, int(np.prod(fs)))
        expect = ocsr.csr_matvec(tcrow, tcol, tval, coef[:, c]) / grid.volume
        got = fields[c].reshape(-1).cpu().numpy()
        np.testing.assert_allclose(got, expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())
        r = ocsr.csr_matvec(crow, col, val, vel[c].reshape(-1))
        np.testing.assert_allclose(rhs[:, c].cpu().numpy(), r, rtol=1e-12, atol=1e-12 * np.abs(r).max())
        power_solid += (coef[:, c] * r).sum()
    # power identity coef·(B u) = vol Σ u·(Bᵀ coef / vol)
    power_fluid = grid.volume * sum((v * f.cpu().numpy()).sum() for v, f in zip(vel, fields))
    assert abs(power_solid - power_fluid) <= 1e-11 * abs(power_solid)
    again = tr.spread(t(coef), A)
    assert all(torch.equal(a, b) for a, b in zip(again, fields))  # fixed per-row order
    # torch view of the operator for reference-typed callers
    dense = A.gather[0].torch().to_dense().cpu().numpy()
    assert dense.shape == (Xn.shape[0], int(np.prod(grid.face_shape(0))))


def test_p1_hash_collisions_duplicates_overflow_and_large_keys():
    """Ports of the reference's table tests (``tests/test_csr_hash_assembly.py:19-57``)."""
    for dtype in (torch.float32, torch.float64):
        colliders = [k for k in range(10000) if ocsr.splitmix_bucket(k, 128) == 3][:40]
        keys = t(colliders * 7 + [987654], torch.int64)
        values = torch.full(keys.shape, .125, device=DEV, dtype=dtype)
        values[-1] = 0
        work = HashWorkspace()
        work.reset(128, values)
        cuda_ib.hash_accumulate(keys, values, work)
        assert work.flag.item() == 0
        occupied = work.keys >= 0
        order = torch.argsort(work.keys[occupied])
        assert work.keys[occupied][order].tolist() == sorted(colliders)
        assert torch.equal(work.values[occupied][order], torch.full((40,), .875, device=DEV, dtype=dtype))
        # the table is the reference's: every key sits in its probe chain from its bucket
        table = work.keys.tolist()
        for s, k in enumerate(table):
            if k >= 0:
                b = ocsr.splitmix_bucket(k, 128)
                assert all(table[(b + i) % 128] != -1 for i in range((s - b) % 128))
        work.reset(8, values)
        cuda_ib.hash_accumulate(torch.arange(20, device=DEV), values[:20], work)
        assert work.flag.item() == 1
        unique = torch.arange(1024, device=DEV, dtype=torch.int64) * 2147483649 + 4294967296
        reps = unique.repeat(128)
        signs = torch.where(torch.arange(128, device=DEV) % 2 == 0, 1., -.5).to(dtype)
        vals = signs.repeat_interleave(len(unique)) * .125
        for _ in range(3):
            work.reset(4096, vals)
            cuda_ib.hash_accumulate(reps, vals, work)
            assert work.flag.item() == 0
            occupied = work.keys >= 0
            order = torch.argsort(work.keys[occupied])
            assert torch.equal(work.keys[occupied][order], unique)
            assert torch.equal(work.values[occupied][order], torch.full((1024,), 128 / 32, device=DEV, dtype=dtype))


def test_p1_cached_contraction_looks_up_and_streams_misses():
    g = golden('p1csr')
    grid = _grid(g)
    X = t(g['block_X'])
    tr = P1CSRTransfer(grid, X, t(g['block_cells']))
    st = tr.prepare_tables(X)
    plans = tr._plans(st)
    c = 1
    shape = grid.face_shape(c)
    full = HashWorkspace()
    full.reset(power_of_two(8 * sum(p[5] for p in plans[c])), st.phi)
    for group, off, low, width, prefix, count in plans[c]:
        cuda_ib.contract(st, group, c, off, low, width, prefix, count, shape, full)
    assert full.flag.item() == 0
    # cached lookup into a table that holds only the first group's keys
    first = HashWorkspace()
    first.reset(full.capacity, st.phi)
    group, off, low, width, prefix, count = plans[c][0]
    cuda_ib.contract(st, group, c, off, low, width, prefix, count, shape, first)
    cached = HashWorkspace()
    cached.reset(full.capacity, st.phi)
    cached.keys.copy_(first.keys)
    miss = MissingStream(torch.empty(1 << 18, dtype=torch.int64, device=DEV), st.phi.new_zeros(1 << 18),
                         torch.zeros(1, dtype=torch.int64, device=DEV))
    for group, off, low, width, prefix, count in plans[c]:
        cuda_ib.contract(st, group, c, off, low, width, prefix, count, shape, cached, cache=miss)
    assert cached.flag.item() == 0
    n = int(miss.missing_count.item())
    assert 0 < n <= miss.missing_keys.numel()
    # cached values + the accumulated misses = the full table
    cuda_ib.hash_accumulate(miss.missing_keys[:n], miss.missing_values[:n], cached)
    def entries(w):
        occ = w.keys >= 0
        order = torch.argsort(w.keys[occ])
        return w.keys[occ][order], w.values[occ][order]
    ka, va = entries(full)
    kb, vb = entries(cached)
    assert torch.equal(ka, kb)
    torch.testing.assert_close(va, vb, rtol=1e-13, atol=1e-16)


def test_p1_fp32_operators_and_budget_errors():
    g = golden('p1csr')
    grid = _grid(g)
    X = t(g['block_X'], torch.float32)
    tr = P1CSRTransfer(grid, X, t(g['block_cells']))
    A = tr.prepare(X)
    ref = P1CSRTransfer(grid, X.double(), t(g['block_cells'])).prepare(X.double())
    for c in range(3):
        dense32 = A.gather[c].torch().to_dense().double()
        dense64 = ref.gather[c].torch().to_dense()
        scale = dense64.abs().max()
        torch.testing.assert_close(dense32, dense64, rtol=3e-5, atol=3e-6 * float(scale))
    small = P1CSRTransfer(grid, X.double(), t(g['block_cells']), max_entries=8)
    with pytest.raises(RuntimeError, match='budget exceeded|probe/budget exceeded'):
        small.prepare(X.double())


def test_p1_precision_form_fp32_transfers_beside_fp64_positions():
    """transfer_dtype=float32 with FP64 positions: rule, tables and contraction
    in FP64, the operator values rounded once to FP32 (equal to the FP64
    values cast), spread and interpolate in FP32 within 2e-6 of the field
    scale of the FP64 oracle; FP64 data is refused."""
    g = golden('p1csr')
    grid = _grid(g)
    Xn, cells = g['block_X'], g['block_cells']
    tr64 = P1CSRTransfer(grid, t(Xn), t(cells))
    tr32 = P1CSRTransfer(grid, t(Xn), t(cells), transfer_dtype=torch.float32)
    A64, A32 = tr64.prepare(t(Xn)), tr32.prepare(t(Xn))
    assert A32.assembly['transfer_dtype'] == 'float32'
    for a, b in zip(A32.gather + A32.spread, A64.gather + A64.spread):
        assert a.val.dtype == torch.float32 and torch.equal(a.val, b.val.float())
        assert torch.equal(a.col, b.col) and torch.equal(a.crow, b.crow)
    rng = np.random.default_rng(9)
    coef = rng.uniform(-1, 1, (Xn.shape[0], 3))
    vel = [rng.standard_normal(grid.face_shape(c)) for c in range(3)]
    fields = tr32.spread(t(coef, torch.float32), A32)
    rhs = tr32.interpolate_rhs(tuple(t(v, torch.float32) for v in vel), A32)
    groups = [(gr.cells.cpu().numpy(), gr.values.cpu().numpy(), gr.weights.cpu().numpy()) for gr in A64.rule.groups]
    base, phi, _ = oib.p2_prepare(Xn, [(c, N) for c, N, _ in groups], grid.origin, grid.spacing, grid.shape)
    for c in range(3):
        fs = grid.face_shape(c)
        _, _, (crow, col, val) = ocsr.assemble(base, phi, groups, c, fs, Xn.shape[0])
        tcrow, tcol, tval = ocsr.csr_transpose(crow, col, val, int(np.prod(fs)))
        expect = ocsr.csr_matvec(tcrow, tcol, tval, coef[:, c]) / grid.volume
        got = fields[c].reshape(-1).double().cpu().numpy()
        np.testing.assert_allclose(got, expect, rtol=0, atol=2e-6 * np.abs(expect).max())
        r = ocsr.csr_matvec(crow, col, val, vel[c].reshape(-1))
        np.testing.assert_allclose(rhs[:, c].double().cpu().numpy(), r, rtol=0, atol=2e-6 * np.abs(r).max())
    with pytest.raises(ValueError, match='float64'):
        tr32.spread(t(coef), A32)


def _table(keys, values):
    from afsi_gpu_b200.p1_csr import HashWorkspace
    ws = HashWorkspace()
    ws.capacity = len(keys)
    ws.keys = t(keys, torch.int64)
    ws.values = t(values)
    ws.flag = torch.zeros((), device=DEV, dtype=torch.int32)
    return ws


def _pattern(cache, matrix, transpose):
    return dict(slots=cache.slots.long().cpu().numpy(), order=cache.transpose_order.long().cpu().numpy(),
                crow=cache.crow.cpu().numpy(), cols=cache.columns.cpu().numpy(),
                tcrow=cache.transpose_crow.cpu().numpy(), tcols=cache.transpose_columns.cpu().numpy(),
                values=matrix.values().cpu().numpy(), reverse=transpose.values().cpu().numpy())


def test_cached_pattern_build_and_merge_match_reference():
    """finish_cached_component on the device against the reference's own
    first build and miss-stream merge (cached.npz): every index array exact,
    values exact (they are read from the same table)."""
    from afsi_gpu_b200.p1_csr import CSRPatternCache, finish_cached_component, numeric_snapshot
    g = golden('cached')
    rows, shape = int(g['rows']), tuple(int(n) for n in g['shape'])
    cache = CSRPatternCache()
    ws = _table(g['table1_keys'], g['table1_values'])
    got = _pattern(cache, *finish_cached_component(ws, cache, rows, shape, 10 ** 6))
    for k in got:
        assert np.array_equal(got[k], g[f'{k}1']), k
    ws2 = _table(g['table2_keys'], g['table2_values'])
    cache.missing_keys = t(g['missing'], torch.int64)
    got = _pattern(cache, *finish_cached_component(ws2, cache, rows, shape, 10 ** 6, missing=len(g['missing'])))
    for k in got:
        assert np.array_equal(got[k], g[f'{k}2']), k
    assert cache.last_sorted_keys == int(g['new_count'])
    m, tr = numeric_snapshot(ws2, cache, rows, shape)
    assert np.array_equal(m.values().cpu().numpy(), g['values2'])
    assert np.array_equal(tr.values().cpu().numpy(), g['reverse2'])
    # nothing new: the snapshot path
    cache.missing_keys = t(g['missing'][:20], torch.int64)
    got = _pattern(cache, *finish_cached_component(ws2, cache, rows, shape, 10 ** 6, missing=20))
    assert cache.last_sorted_keys == 0 and np.array_equal(got['slots'], g['slots2'])


def test_cached_pattern_large_merge_against_oracle():
    from afsi_gpu_b200.p1_csr import CSRPatternCache, HashWorkspace, finish_cached_component, hash_accumulate
    rng = np.random.default_rng(9)
    rows, shape = 5000, (24, 20, 16)
    nf = int(np.prod(shape))
    ws = HashWorkspace()
    ws.reset(1 << 16, torch.zeros(1, device=DEV, dtype=torch.float64))
    k1 = rng.integers(0, rows * nf, 20000)
    hash_accumulate(t(k1, torch.int64), t(rng.standard_normal(len(k1))), ws)
    assert int(ws.flag.item()) == 0
    cache = CSRPatternCache()
    finish_cached_component(ws, cache, rows, shape, 10 ** 7)
    first = ocsr.finish_cached(ws.keys.cpu().numpy(), ws.values.cpu().numpy(), rows, nf)
    assert np.array_equal(cache.slots.long().cpu().numpy(), first['slots'])
    old_keys = ws.keys.cpu().numpy()[first['slots']]
    k2 = np.concatenate((rng.integers(0, rows * nf, 4000), old_keys[rng.integers(0, len(old_keys), 2000)]))
    hash_accumulate(t(k2, torch.int64), t(rng.standard_normal(len(k2))), ws)
    cache.missing_keys = t(k2, torch.int64)
    m, tr = finish_cached_component(ws, cache, rows, shape, 10 ** 7, missing=len(k2))
    ref = ocsr.finish_cached(ws.keys.cpu().numpy(), ws.values.cpu().numpy(), rows, nf, old=first, missing=k2)
    got = _pattern(cache, m, tr)
    for k in got:
        assert np.array_equal(got[k], ref[k]), k
    # the merged pattern equals a first build of the same table
    again = CSRPatternCache()
    finish_cached_component(ws, again, rows, shape, 10 ** 7)
    assert torch.equal(again.slots, cache.slots) and torch.equal(again.transpose_order, cache.transpose_order)
    assert torch.equal(again.crow, cache.crow) and torch.equal(again.transpose_crow, cache.transpose_crow)
