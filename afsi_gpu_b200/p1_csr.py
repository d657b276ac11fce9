"""P1 quadrature IB contracted to paired CSR operators on the B200 kernels.

Mirrors the CUDA-contraction hash backend of the reference's
``AssembledP1Transfer`` (``mac/assembled_transfer.py:151-216``,
``mac/hash_transfer_assembly.py:26-165``): for component c,
B_c[node, face] = Σ_q W[q] N[q,a] φ_c(face, x_q).  The spread response is
Bᵀ_c·coefficient / cell volume and the interpolation right-hand side is
B_c·u_c; the consistent-mass solve that the reference wraps around them is
outside this hot path (the caller supplies the solved coefficient).

Per prepare and component: a support-box plan per quadrature group
(``afsi_b200_p1_component_plan``), the contraction into a SplitMix64 hash
(``afsi_b200_hash_contract``, the reference's table format and probe rules),
retry with a doubled table on overflow, and the table-to-CSR conversion of B
and Bᵀ (``afsi_b200_hash_csr``).  Host reads are batched: one for the site
counts of every group and component, one for the three overflow flags, one for
the three entry counts.  Responses are CSR SpMV launches
(``afsi_b200_csr_spmv``), summed per row in a fixed order.

``contract`` and ``hash_accumulate`` keep the signatures of
``mac/cuda_ib.py:93-112``.
"""
from dataclasses import dataclass
from math import prod
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code
from .quadrature import RuleBuilder, InteractionRule
from .p2_cuda_transfer import SharedAdaptiveStencil


def power_of_two(n):
    return 1 << max(0, (int(n) - 1).bit_length())


@dataclass
class HashWorkspace:
    """``mac/hash_transfer_assembly.py:26-53``: reusable bounded scratch."""
    capacity: int = 0
    keys: torch.Tensor = None
    values: torch.Tensor = None
    flag: torch.Tensor = None
    allocations: int = 0
    reuses: int = 0

    def reset(self, capacity, like):
        if capacity < 1 or capacity & (capacity - 1):
            raise ValueError('power-of-two hash capacity required')
        if (self.capacity != capacity or self.values is None or self.values.device != like.device
                or self.values.dtype != like.dtype):
            self.keys = torch.empty(capacity, device=like.device, dtype=torch.int64)
            self.values = torch.empty(capacity, device=like.device, dtype=like.dtype)
            self.flag = torch.empty((), device=like.device, dtype=torch.int32)
            self.capacity = capacity
            self.allocations += 1
        else:
            self.reuses += 1
        self.keys.fill_(-1)
        self.values.zero_()
        self.flag.zero_()

    @property
    def storage_bytes(self):
        return self.capacity * (8 + self.values.element_size()) + 4 if self.values is not None else 0


@dataclass
class MissingStream:
    """Miss stream of a cached contraction (``cached_contract_``)."""
    missing_keys: torch.Tensor
    missing_values: torch.Tensor
    missing_count: torch.Tensor


def _check_table(workspace):
    for t in (workspace.keys, workspace.values, workspace.flag):
        _lib.require_cuda(t)
    if workspace.keys.dtype != torch.int64 or workspace.flag.dtype != torch.int32:
        raise RuntimeError('IB hash keys must be int64 and the flag int32')
    if workspace.keys.numel() != workspace.values.numel() or workspace.keys.numel() & (workspace.keys.numel() - 1):
        raise RuntimeError('power-of-two hash capacity required')


def contract(stencil, group, component, offset, low, width, prefix, count, face_shape, workspace, cache=None):
    """``cuda_ib.contract`` (``mac/cuda_ib.py:93-106``): add the four nodal
    sums of every box site of the group's cells into the workspace table."""
    _check_table(workspace)
    shared = getattr(stencil, 'layout', None) == 'shared'
    base, phi = stencil.base, stencil.phi
    dt = workspace.values.dtype
    if phi.dtype != dt or group.values.dtype != dt or group.weights.dtype != dt:
        raise RuntimeError('IB contraction requires matching floating dtypes')
    ny, nz = face_shape[1], face_shape[2]
    nf = face_shape[0] * ny * nz
    args = (ptr(base), ptr(phi), ptr(group.values), ptr(group.weights), ptr(group.cells), ptr(low), ptr(width),
            ptr(prefix))
    tail = (base.shape[1], offset, group.cells.shape[0], group.values.shape[0], int(count), int(component), ny, nz,
            nf, int(shared), dtype_code(dt), stream(base.device))
    if cache is None:
        call('afsi_b200_hash_contract', *args, ptr(workspace.keys), ptr(workspace.values), ptr(workspace.flag),
             workspace.capacity, *tail)
    else:
        call('afsi_b200_cached_contract', *args, ptr(workspace.keys), ptr(workspace.values), ptr(workspace.flag),
             workspace.capacity, ptr(cache.missing_keys), ptr(cache.missing_values), ptr(cache.missing_count),
             cache.missing_keys.numel(), *tail)


def hash_accumulate(keys, values, workspace):
    """``cuda_ib.hash_accumulate`` (``mac/cuda_ib.py:109-112``)."""
    _check_table(workspace)
    _lib.require_cuda(keys)
    if keys.dtype != torch.int64 or values.dtype != workspace.values.dtype or keys.numel() != values.numel():
        raise RuntimeError('IB entry stream shape mismatch')
    keys, values = keys.contiguous(), values.contiguous()
    call('afsi_b200_hash_accumulate', ptr(keys), ptr(values), keys.numel(), ptr(workspace.keys),
         ptr(workspace.values), ptr(workspace.flag), workspace.capacity, dtype_code(values.dtype),
         stream(keys.device))


@dataclass(frozen=True)
class CSR:
    """One assembled operator: CSR arrays on the device (entries [0, nnz))."""
    crow: torch.Tensor
    col: torch.Tensor
    val: torch.Tensor
    shape: tuple

    @property
    def nnz(self):
        return self.col.numel()

    def torch(self):
        """The operator as a ``torch.sparse_csr_tensor`` (the reference's type)."""
        return torch.sparse_csr_tensor(self.crow, self.col, self.val, self.shape, check_invariants=False)

    def matvec(self, x, out, *, x_stride=1, out_stride=1, divisor=1.):
        call('afsi_b200_csr_spmv', ptr(self.crow), ptr(self.col), ptr(self.val), self.shape[0], self.nnz, ptr(x),
             x_stride, ptr(out), out_stride, float(divisor), dtype_code(self.val.dtype), stream(self.val.device))
        return out


@dataclass(frozen=True)
class AssembledStencil:
    """``mac/assembled_transfer.py:15-27``: B_c (gather) and Bᵀ_c (spread)."""
    gather: tuple
    spread: tuple
    rule: InteractionRule
    assembly: dict

    @property
    def storage_bytes(self):
        return sum(t.numel() * t.element_size() for a in self.gather + self.spread for t in (a.crow, a.col, a.val))


class P1CSRTransfer:
    """Grid/quadrature state of the assembled P1 transfer (no mass solve).

    ``prepare(x)`` builds the adaptive rule and the shared face/centre tables
    (``afsi_b200_p1_prepare``) and contracts them to CSR; ``spread`` and
    ``interpolate_rhs`` apply the operators."""

    def __init__(self, grid, X, cells, *, point_density=2., max_order=8, max_points=12000000,
                 max_entries=32000000, transfer_dtype=None):
        if cells.dim() != 2 or cells.shape[1] != 4:
            raise ValueError('P1 CSR transfer requires four-node tetrahedra')
        if type(max_entries) is not int or max_entries < 1:
            raise ValueError('positive CSR entry budget required')
        _lib.require_cuda(X)
        # precision form: FP64 positions, tables and contraction; the assembled
        # operator values stored once per prepare in FP32 and applied in FP32
        self.transfer_dtype = X.dtype if transfer_dtype is None else transfer_dtype
        if self.transfer_dtype != X.dtype and not (X.dtype == torch.float64 and self.transfer_dtype == torch.float32):
            raise ValueError('FP32 transfers are supported beside FP64 positions only')
        self.grid = grid
        self.node_count = X.shape[0]
        self.cells = cells.contiguous()
        self.max_entries = max_entries
        self.rules = RuleBuilder(X, self.cells, grid, point_density=point_density, max_order=max_order,
                                 max_points=max_points)
        self.hash_workspaces = tuple(HashWorkspace() for _ in range(3))
        self._plan_scratch = None
        self._csr_scratch = {}
        self.csr_builds = 0

    # -- tables
    def prepare_tables(self, x):
        _lib.require_cuda(x)
        x = x.contiguous()
        rule = self.rules(x)
        total = rule.point_count
        base = torch.empty((2, total, 3), device=x.device, dtype=torch.int64)
        phi = x.new_empty((2, total, 3, 4))
        word = _lib.status_word(x.device)
        word.zero_()
        g = self.grid
        limits = [n - 2 for n in g.shape]
        offset = 0
        for group in rule.groups:
            call('afsi_b200_p1_prepare', ptr(x), x.shape[0], ptr(group.cells), group.cells.shape[0],
                 ptr(group.values), group.values.shape[0], _lib.doubles(g.origin), _lib.doubles(g.spacing),
                 _lib.doubles(limits), ptr(base), ptr(phi), total, offset, ptr(word), dtype_code(x.dtype),
                 stream(x.device))
            offset += group.weights.numel()
        flags = int(word.item())
        if flags:
            word.zero_()
            if flags & _lib.FLAG_INDEX:
                raise RuntimeError('P1 connectivity outside the node range')
            raise ValueError('MAC IB support reaches a wall or is nonfinite; enlarge/refine the fluid box')
        return SharedAdaptiveStencil(base, phi, rule)

    # -- assembly
    def _plans(self, stencil):
        """low/width/prefix of every group and component; one host read of the counts."""
        rule = stencil.rule
        device = stencil.base.device
        groups, offset = [], 0
        for group in rule.groups:
            groups.append((group, offset))
            offset += group.weights.numel()
        largest = max(g.cells.shape[0] for g, _ in groups)
        need = _lib.load().afsi_b200_p1_plan_scratch_bytes(largest)
        if self._plan_scratch is None or self._plan_scratch.numel() < need or self._plan_scratch.device != device:
            self._plan_scratch = torch.empty(need, dtype=torch.uint8, device=device)
        plans = [[] for _ in range(3)]
        for c in range(3):
            for group, off in groups:
                E = group.cells.shape[0]
                low = torch.empty((E, 3), dtype=torch.int64, device=device)
                width = torch.empty((E, 3), dtype=torch.int64, device=device)
                prefix = torch.empty(E + 1, dtype=torch.int64, device=device)
                call('afsi_b200_p1_component_plan', ptr(stencil.base), stencil.base.shape[1], off, E,
                     group.values.shape[0], c, 1, ptr(low), ptr(width), ptr(prefix), ptr(self._plan_scratch),
                     self._plan_scratch.numel(), stream(device))
                plans[c].append([group, off, low, width, prefix, None])
        counts = torch.stack([p[4][-1] for c in range(3) for p in plans[c]]).tolist()
        k = 0
        for c in range(3):
            for p in plans[c]:
                p[5] = int(counts[k])
                k += 1
        return plans

    def _csr_scratch_for(self, capacity, like):
        key = (capacity, like.dtype, like.device)
        if key not in self._csr_scratch:
            need = _lib.load().afsi_b200_hash_csr_scratch_bytes(capacity, dtype_code(like.dtype))
            self._csr_scratch = {key: torch.empty(need, dtype=torch.uint8, device=like.device)}
        return self._csr_scratch[key]

    @torch.no_grad()
    def assemble_stencil(self, stencil):
        """B_c and Bᵀ_c for c = 0, 1, 2 (``AssembledP1Transfer.assemble_stencil``
        with the hash assembly and the CUDA contraction)."""
        like = stencil.rule.groups[0].weights
        plans = self._plans(stencil)
        limit = power_of_two(2 * self.max_entries)
        shapes = [self.grid.face_shape(c) for c in range(3)]
        raw = [4 * sum(p[5] for p in plans[c]) for c in range(3)]
        attempts = [0, 0, 0]
        pending = [0, 1, 2]
        while pending:
            for c in pending:
                w = self.hash_workspaces[c]
                if attempts[c] == 0:
                    capacity = min(limit, max(w.capacity, power_of_two(max(128, raw[c] // 8))))
                else:
                    capacity = min(limit, 2 * w.capacity)
                w.reset(capacity, like)
                attempts[c] += 1
                for group, off, low, width, prefix, count in plans[c]:
                    contract(stencil, group, c, off, low, width, prefix, count, shapes[c], w)
            flags = torch.stack([self.hash_workspaces[c].flag for c in pending]).tolist()
            failed = [c for c, f in zip(pending, flags) if f]
            for c in failed:
                if self.hash_workspaces[c].capacity >= limit:
                    raise RuntimeError('assembled IB hash probe/budget exceeded; raise max_entries')
            pending = failed
        results = []
        infos = []
        for c in range(3):
            w = self.hash_workspaces[c]
            nf = prod(shapes[c])
            cap = w.capacity
            crow = torch.empty(self.node_count + 1, dtype=torch.int64, device=like.device)
            col = torch.empty(cap, dtype=torch.int64, device=like.device)
            val = like.new_empty(cap)
            t_crow = torch.empty(nf + 1, dtype=torch.int64, device=like.device)
            t_col = torch.empty(cap, dtype=torch.int64, device=like.device)
            t_val = like.new_empty(cap)
            info = torch.empty(2, dtype=torch.int64, device=like.device)
            scratch = self._csr_scratch_for(cap, like)
            call('afsi_b200_hash_csr', ptr(w.keys), ptr(w.values), cap, self.node_count, nf, ptr(crow), ptr(col),
                 ptr(val), ptr(t_crow), ptr(t_col), ptr(t_val), ptr(info), ptr(scratch), scratch.numel(),
                 dtype_code(like.dtype), stream(like.device))
            results.append((crow, col, val, t_crow, t_col, t_val, nf))
            infos.append(info)
        info = torch.stack(infos).tolist()
        gather, spread, stats, remaining = [], [], [], self.max_entries
        for c, ((crow, col, val, t_crow, t_col, t_val, nf), (nnz, bad)) in enumerate(zip(results, info)):
            if nnz > remaining:
                raise RuntimeError('assembled IB entry budget exceeded; no hash entries were truncated')
            if bad:
                raise FloatingPointError('invalid hash IB entries: nonfinite values or out-of-range keys')
            remaining -= nnz
            gather.append(CSR(crow, col[:nnz], val[:nnz], (self.node_count, nf)))
            spread.append(CSR(t_crow, t_col[:nnz], t_val[:nnz], (nf, self.node_count)))
            w = self.hash_workspaces[c]
            stats.append(dict(raw_cell_entries=raw[c], nnz=nnz, hash_capacity=w.capacity, hash_attempts=attempts[c],
                              hash_workspace_bytes=w.storage_bytes, hash_workspace_allocations=w.allocations,
                              hash_workspace_reuses=w.reuses, raw_entries_materialized=False, unique_key_sorts=1,
                              duplicate_merge_sorts=0))
        self.csr_builds += 1
        return AssembledStencil(tuple(gather), tuple(spread), stencil.rule,
                                dict(components=stats, total_nnz=sum(s['nnz'] for s in stats),
                                     max_entries=self.max_entries, assembly_backend='hash',
                                     contraction_backend='cuda', builder='b200-cell-warp+device-hash+radix-csr'))

    def prepare(self, x):
        st = self.assemble_stencil(self.prepare_tables(x))
        if st.gather[0].val.dtype == self.transfer_dtype:
            return st
        cast = lambda ops: tuple(CSR(a.crow, a.col, a.val.to(self.transfer_dtype), a.shape) for a in ops)
        return AssembledStencil(cast(st.gather), cast(st.spread), st.rule,
                                dict(st.assembly, transfer_dtype=str(self.transfer_dtype).replace('torch.', '')))

    def _check_dtype(self, t, stencil):
        if t.dtype != stencil.gather[0].val.dtype:
            raise ValueError(f'P1 CSR transfer in {stencil.gather[0].val.dtype} got {t.dtype} data')

    # -- responses
    def spread(self, coefficient, stencil):
        """Face densities Bᵀ_c·coefficient[:,c] / volume (the reference's
        ``spread`` after its mass solve, ``assembled_transfer.py:195-202``)."""
        _lib.require_cuda(coefficient)
        coefficient = coefficient.contiguous()
        if coefficient.shape != (self.node_count, 3):
            raise ValueError('P1 CSR spread expects nodal coefficients (N,3)')
        self._check_dtype(coefficient, stencil)
        out = []
        for c, BT in enumerate(stencil.spread):
            field = coefficient.new_empty(self.grid.face_shape(c))
            BT.matvec(coefficient[:, c:], field, x_stride=3, divisor=self.grid.volume)
            out.append(field)
        return tuple(out)

    def interpolate_rhs(self, velocity, stencil):
        """B_c·u_c per component into (N,3) (the reference's ``interpolate``
        before its mass solve, ``assembled_transfer.py:204-212``)."""
        out = None
        for c, (B, u) in enumerate(zip(stencil.gather, velocity)):
            _lib.require_cuda(u)
            self._check_dtype(u, stencil)
            u = u.contiguous()
            if out is None:
                out = u.new_empty((self.node_count, 3))
            B.matvec(u, out[:, c:], out_stride=3)
        return out


# ------------------------------------------------------------ cached pattern

class PatternBudgetExceeded(RuntimeError):
    """``mac/cached_transfer_assembly.py:15-16``."""


@dataclass
class CSRPatternCache:
    """The fields of ``CSRPatternCache`` (``mac/cached_transfer_assembly.py:19-69``)
    that the pattern maintenance reads and writes."""
    slots: torch.Tensor = None
    transpose_order: torch.Tensor = None
    crow: torch.Tensor = None
    columns: torch.Tensor = None
    transpose_crow: torch.Tensor = None
    transpose_columns: torch.Tensor = None
    missing_keys: torch.Tensor = None
    missing_values: torch.Tensor = None
    missing_count: torch.Tensor = None
    missing_capacity: int = 0
    rebuilds: int = 0
    pattern_shape: tuple = None
    last_sorted_keys: int = 0
    total_sorted_keys: int = 0

    @property
    def nnz(self):
        return 0 if self.slots is None else len(self.slots)


def finish_cached_component(workspace, cache, node_count, shape, max_entries, *, missing=None):
    """``finish_cached_component`` (``mac/cached_transfer_assembly.py:97-175``)
    on the device: the first build from the occupied table keys, or the merge
    of the keys of the miss stream (``missing`` of them) that the pattern
    lacks into the slot order, the transpose order and both row-pointer
    arrays (``afsi_b200_cache_new_keys`` then ``afsi_b200_cache_merge``; one
    host read of the new-key count between them, as in the reference).
    Works on the reference's workspace and cache objects or on the ones of
    this module; returns (B, Bᵀ) as CSR tensors sharing the cache's indices."""
    keys_t, values_t = workspace.keys, workspace.values
    _lib.require_cuda(keys_t)
    dev = keys_t.device
    nf = prod(shape)
    cap = int(workspace.capacity)
    limit = nf * node_count
    s = stream(dev)
    lib = _lib.load()
    if missing is None:
        scratch = torch.empty(int(lib.afsi_b200_cache_scratch_bytes(cap, 0, 0, node_count, nf)), device=dev,
                              dtype=torch.uint8)
        sorted_keys = torch.empty(cap, device=dev, dtype=torch.int64)
        sorted_slots = torch.empty(cap, device=dev, dtype=torch.int64)
        count = torch.zeros(1, device=dev, dtype=torch.int64)
        call('afsi_b200_cache_new_keys', ptr(keys_t), cap, None, 0, None, 0, limit, ptr(sorted_keys),
             ptr(sorted_slots), ptr(count), ptr(scratch), scratch.numel(), s)
        k = int(count.item())
        if k > max_entries:
            raise PatternBudgetExceeded('cached IB union exceeds entry budget')
        new_keys, new_slots = sorted_keys[:k], sorted_slots[:k]
        old = None
        nnz_old = 0
    else:
        old_slots = cache.slots.to(torch.int64)
        nnz_old = len(old_slots)
        scratch = torch.empty(int(lib.afsi_b200_cache_scratch_bytes(cap, nnz_old, int(missing), node_count, nf)),
                              device=dev, dtype=torch.uint8)
        new_buf = torch.empty(max(int(missing), 1), device=dev, dtype=torch.int64)
        count = torch.zeros(1, device=dev, dtype=torch.int64)
        call('afsi_b200_cache_new_keys', ptr(keys_t), cap, ptr(old_slots), nnz_old, ptr(cache.missing_keys),
             int(missing), limit, ptr(new_buf), None, ptr(count), ptr(scratch), scratch.numel(), s)
        k = int(count.item())
        if nnz_old + k > max_entries:
            raise PatternBudgetExceeded('cached IB union exceeds entry budget')
        if k == 0:
            cache.last_sorted_keys = 0
            return numeric_snapshot(workspace, cache, node_count, shape)
        new_keys, new_slots = new_buf[:k], None
        old = (old_slots, cache.transpose_order.to(torch.int64), cache.crow, cache.transpose_crow)
    n = nnz_old + k
    out = dict(slots=torch.empty(n, device=dev, dtype=torch.int64), order=torch.empty(n, device=dev, dtype=torch.int64),
               crow=torch.empty(node_count + 1, device=dev, dtype=torch.int64),
               columns=torch.empty(n, device=dev, dtype=torch.int64),
               tcrow=torch.empty(nf + 1, device=dev, dtype=torch.int64),
               tcolumns=torch.empty(n, device=dev, dtype=torch.int64),
               values=torch.empty(n, device=dev, dtype=values_t.dtype),
               reverse=torch.empty(n, device=dev, dtype=values_t.dtype))
    status = torch.zeros(1, device=dev, dtype=torch.int32)
    call('afsi_b200_cache_merge', ptr(keys_t), ptr(values_t), cap, *(ptr(t) for t in (old or (None,) * 4)), nnz_old,
         ptr(new_keys), ptr(new_slots), k, node_count, nf, ptr(out['slots']), ptr(out['order']), ptr(out['crow']),
         ptr(out['columns']), ptr(out['tcrow']), ptr(out['tcolumns']), ptr(out['values']), ptr(out['reverse']),
         ptr(status), ptr(scratch), scratch.numel(), dtype_code(values_t.dtype), s)
    word = int(status.item())
    if word & _lib.FLAG_OVERFLOW:
        raise RuntimeError('cached IB slot lookup failed after completed insertion')
    if word & (_lib.FLAG_INDEX | _lib.FLAG_SUPPORT):
        raise FloatingPointError('invalid cached IB entries: nonfinite values or out-of-range keys')
    mapping = torch.int32 if max(cap, n) < 2 ** 31 else torch.int64
    cache.slots, cache.transpose_order = out['slots'].to(mapping), out['order'].to(mapping)
    cache.crow, cache.columns = out['crow'], out['columns']
    cache.transpose_crow, cache.transpose_columns = out['tcrow'], out['tcolumns']
    cache.pattern_shape = (node_count, *shape)
    cache.last_sorted_keys = k
    cache.total_sorted_keys += k
    cache.rebuilds += 1
    matrix = torch.sparse_csr_tensor(out['crow'], out['columns'], out['values'], (node_count, nf),
                                     check_invariants=False)
    transpose = torch.sparse_csr_tensor(out['tcrow'], out['tcolumns'], out['reverse'], (nf, node_count),
                                        check_invariants=False)
    return matrix, transpose


def numeric_snapshot(workspace, cache, node_count, shape, *, validate=True, values=None):
    """``numeric_snapshot`` (``mac/cached_transfer_assembly.py:161-175``): the
    pattern's values read from the table in key and in transpose order."""
    dev = workspace.keys.device
    nf = prod(shape)
    n = cache.nnz
    slots = cache.slots.to(torch.int64)
    order = cache.transpose_order.to(torch.int64)
    vals = torch.empty(n, device=dev, dtype=workspace.values.dtype)
    rev = torch.empty_like(vals)
    status = torch.zeros(1, device=dev, dtype=torch.int32)
    call('afsi_b200_cache_values', ptr(workspace.values), ptr(slots), ptr(order), n, ptr(vals), ptr(rev),
         ptr(status), dtype_code(vals.dtype), stream(dev))
    if validate and int(status.item()):
        raise FloatingPointError('invalid cached IB entries: nonfinite values')
    matrix = torch.sparse_csr_tensor(cache.crow, cache.columns, vals, (node_count, nf), check_invariants=False)
    transpose = torch.sparse_csr_tensor(cache.transpose_crow, cache.transpose_columns, rev, (nf, node_count),
                                        check_invariants=False)
    return matrix, transpose
