"""Host side of the batched V-cycles (no GPU): the table that
``afsi_b200_mg_batch_table`` writes for a batch of channel plans.

The plans carry fake, distinct buffer addresses (nothing is dereferenced on
the host).  The table is decoded here with the layout of mg.cu's BatchLevel,
BatchStart and BatchCoarse for float levels and double coarse inverses, and
checked: every tile of every launched level appears exactly once in its
depth's block map, each entry names its instance's buffers (the pre-smoothed
iterate and the coarser final iterate by the smooth parity), every instance
has one start job and one coarse job, coarse jobs largest first.
"""
import ctypes
import numpy as np
import pytest
from afsi_gpu_b200 import _lib
from afsi_gpu_b200.multigrid import _levels

TILE_Y, TILE_X, LOCAL_BITS = 32, 32, 21
LV = np.dtype([('nx', '<i4'), ('ny', '<i4'), ('nz', '<i4'), ('pad', '<i4'), ('n', '<i8'), ('h2', '<f4', 3),
               ('ih2', '<f4', 3)])
LEVEL = np.dtype([('w', '<f4', 64), ('L', LV), ('C', LV), ('p', '<u8'), ('q', '<u8'), ('r', '<u8'), ('rc', '<u8'),
                  ('down', '<u8'), ('corr', '<u8')])
START = np.dtype([('src', '<u8'), ('r', '<u8'), ('p', '<u8'), ('nx', '<i4'), ('ny', '<i4')])
COARSE = np.dtype([('lv', LV, _lib.MAX_LEVELS), ('first', '<i4'), ('last', '<i4'), ('rhs', '<u8'),
                   ('p_start', '<u8'), ('p_out', '<u8'), ('cinv', '<u8')])


def a16(v):
    return (v + 15) // 16 * 16


def tiles(nx, ny):
    return -(-ny // TILE_Y) * -(-nx // TILE_X)


def coarse_start(shapes):
    """First level run in one CTA: <= 4096 cells and its arrays (with every
    coarser level's and 64 table entries per level) in 200 KB of FP32."""
    cells = [nx * ny for nx, ny in shapes]
    for l in range(len(shapes)):
        if cells[l] <= 4096 and (sum(cells[l:]) * 3 + 64 * (len(shapes) - l)) * 4 <= 200 * 1024:
            return l
    return len(shapes) - 1


def fake_plans(grid_shapes, smooth):
    plans, addr = [], [1 << 32]

    def new():
        addr[0] += 1 << 20
        return addr[0]
    for nx, ny in grid_shapes:
        shapes, spacings = _levels((nx, ny), (4. / nx, 1. / ny))
        plan = _lib.MGPlan()
        plan.dim, plan.bc, plan.levels, plan.smooth = 2, _lib.BC_CHANNEL, len(shapes), smooth
        plan.dtype, plan.coarse_dtype, plan.smoother = _lib.F32, _lib.F64, 0
        for l, (s, h) in enumerate(zip(shapes, spacings)):
            L = plan.level[l]
            for a in range(3):
                L.shape[a] = (list(s) + [1])[a]
                L.h2[a] = (list(h) + [1.])[a] ** 2
                L.inv_h2[a] = 1 / L.h2[a]
            L.p, L.ping, L.rhs = new(), new(), new()
        plan.coarse_inverse, plan.scratch = new(), new()
        plans.append((plan, shapes))
    return plans


def plan_array(plans):
    return (ctypes.POINTER(_lib.MGPlan) * len(plans))(*[ctypes.pointer(p) for p, _ in plans])


@pytest.mark.parametrize('smooth', [4, 3])
def test_batch_table_covers_every_tile_once(smooth):
    grid_shapes = [(512, 128), (128, 32), (384, 96), (16, 4), (256, 64), (512, 128), (72, 8)]
    plans = fake_plans(grid_shapes, smooth)
    lib = _lib.load()
    arr = plan_array(plans)
    sources = [(1 << 44) + 4096 * i for i in range(len(plans))]
    src = (ctypes.c_void_p * len(plans))(*sources)
    nbytes = lib.afsi_b200_mg_batch_table_bytes(arr, len(plans))
    assert nbytes > 0
    host = np.zeros(nbytes, np.uint8)
    _lib.call('afsi_b200_mg_batch_table', arr, len(plans), src, host.ctypes.data, nbytes)

    starts = [coarse_start(shapes) for _, shapes in plans]
    assert starts == [2, 0, 2, 0, 1, 2, 0]
    off = 0
    for d in range(max(starts)):
        members = [i for i, s in enumerate(starts) if s > d]
        lv = np.frombuffer(host, LEVEL, len(members), off)
        off = a16(off + len(members) * LEVEL.itemsize)
        bl = sum(tiles(*plans[i][1][d]) for i in members)
        ml = np.frombuffer(host, '<u4', bl, off)
        off = a16(off + 4 * bl)
        bc = sum(tiles(*plans[i][1][d + 1]) for i in members)
        mc = np.frombuffer(host, '<u4', bc, off)
        off = a16(off + 4 * bc)
        for k, i in enumerate(members):
            plan, shapes = plans[i]
            P, Q = (lambda l: plan.level[l].p), (lambda l: plan.level[l].ping)
            e = lv[k]
            assert (e['L']['nx'], e['L']['ny'], e['L']['nz']) == (*shapes[d], 1)
            # omega/diag of an interior cell (class 48: 2D, both z bits), the
            # channel diagonal summed x then y in FP32, one division
            ihx, ihy = e['L']['ih2'][0], e['L']['ih2'][1]
            d_int = ((np.float32(0) + ihx + ihx) + ihy) + ihy
            assert e['w'][48] == np.float32(2.0 / 3.0) / d_int
            assert (e['C']['nx'], e['C']['ny']) == shapes[d + 1] and e['C']['n'] == np.prod(shapes[d + 1])
            assert (e['p'], e['q'], e['r'], e['rc']) == (P(d), Q(d), plan.level[d].rhs, plan.level[d + 1].rhs)
            assert e['down'] == (P(d) if smooth % 2 == 0 else Q(d))
            assert e['corr'] == (P(d + 1) if (d + 1 >= starts[i] or smooth % 2 == 0) else Q(d + 1))
            for m, shape in ((ml, shapes[d]), (mc, shapes[d + 1])):
                own = np.sort(m[(m >> LOCAL_BITS) == k] & ((1 << LOCAL_BITS) - 1))
                assert np.array_equal(own, np.arange(tiles(*shape)))
        assert np.all((ml >> LOCAL_BITS) < len(members)) and np.all((mc >> LOCAL_BITS) < len(members))
    st = np.frombuffer(host, START, len(plans), off)
    off = a16(off + len(plans) * START.itemsize)
    total = sum(tiles(*shapes[0]) for _, shapes in plans)
    ms = np.frombuffer(host, '<u4', total, off)
    off = a16(off + 4 * total)
    for i, (plan, shapes) in enumerate(plans):
        assert (st[i]['src'], st[i]['r'], st[i]['p']) == (sources[i], plan.level[0].rhs, plan.level[0].p)
        assert (st[i]['nx'], st[i]['ny']) == shapes[0]
        own = np.sort(ms[(ms >> LOCAL_BITS) == i] & ((1 << LOCAL_BITS) - 1))
        assert np.array_equal(own, np.arange(tiles(*shapes[0])))
    co = np.frombuffer(host, COARSE, len(plans), off)
    assert a16(off + len(plans) * COARSE.itemsize) == nbytes
    seen, smem = [], []
    for j in co:
        i = next(i for i, (p, _) in enumerate(plans) if p.coarse_inverse == j['cinv'])
        plan, shapes = plans[i]
        f = starts[i]
        assert (j['first'], j['last']) == (f, len(shapes) - 1)
        assert j['rhs'] == plan.level[f].rhs and j['p_out'] == plan.level[f].p
        assert j['p_start'] == (plan.level[0].p if f == 0 else 0)
        seen.append(i)
        smem.append(sum(nx * ny for nx, ny in shapes[f:]) * 3 + 64 * (len(shapes) - f))
    assert sorted(seen) == list(range(len(plans)))
    assert smem == sorted(smem, reverse=True)


def test_batch_rejects_mixed_plans():
    plans = fake_plans([(128, 32), (256, 64)], 4)
    lib = _lib.load()
    arr = plan_array(plans)
    plans[1][0].smooth = 2
    assert lib.afsi_b200_mg_batch_table_bytes(arr, 2) == -1
    plans[1][0].smooth = 4
    plans[1][0].smoother = 1
    assert lib.afsi_b200_mg_batch_table_bytes(arr, 2) == -1
    plans[1][0].smoother = 0
    plans[1][0].bc = _lib.BC_PERIODIC
    assert lib.afsi_b200_mg_batch_table_bytes(arr, 2) == -1
    plans[1][0].bc = _lib.BC_CHANNEL
    assert lib.afsi_b200_mg_batch_table_bytes(arr, 2) > 0
    host = np.zeros(8, np.uint8)
    with pytest.raises(RuntimeError, match='table needs'):
        _lib.call('afsi_b200_mg_batch_table', arr, 2, None, host.ctypes.data, 8)
