"""P2 quadrature IB transfer on the B200 kernels.

Module functions keep the signatures of ``afsi_torch/mac/p2_cuda_transfer.py``
(``prepare(transfer, x, rule, *, buffers=None)``, ``spread(transfer,
coefficient, stencil)``, ``assemble_velocity(transfer, velocity, stencil)``)
and the semantics of the ``p2_prepare_ / p2_spread_ / p2_gather_assemble_``
operators (``mac/csrc/p2_transfer.cpp:66-74``): shared face/centre tables
(2,T,3)/(2,T,3,4), one launch per quadrature group, spreads accumulate into
fresh zeroed fields, the nodal right-hand side accumulates into zeros, and a
support violation raises ``ValueError`` after the prepare.

``P2Transfer`` supplies what those functions read from the reference
``AdaptiveFETransfer`` (grid, origin/spacing/limits, diagonal, rule) without
the consistent-mass solve, which is outside this hot path.  Its
``deterministic=True`` mode assembles through element-local sums and a fixed
node CSR instead of atomics (bitwise reproducible ``assemble_velocity``).
``transfer_dtype=torch.float32`` beside FP64 positions is the precision form:
positions, bases and weights are formed in FP64 (``afsi_b200_fe_prepare_mixed``,
so the bases are the FP64 bases), the weight tables, rule tables and the
transfers are FP32.

Table-free form (``P2Transfer.prepare_table_free``, ``TableFreeStencil``): the
rule only, no stencil tables; ``spread`` / ``assemble_velocity`` then form each
point's position, bases and weights inside the transfer kernels
(``afsi_b200_fe_fused_spread/_gather``) with the prepare's arithmetic, so the
results equal the table-based ones up to the order of the atomic additions.
Support and connectivity violations are flagged into the stencil's status
word by the transfers and raised by ``confirm``.  ``P1Transfer`` is the
matrix-free P1 element transfer (``mac/adaptive_cell.py:22-83``) on the same
kernels with four-node cells.
"""
from dataclasses import dataclass
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code
from .quadrature import RuleBuilder, InteractionRule


@dataclass
class DeferredStencil:
    """Tables prepared with the cached rule before the rule was checked
    (``P2Transfer.prepare_deferred``): ``stencil`` is usable at once;
    ``P2Transfer.confirm`` settles it.  Until then a point outside the support
    may have rows with base -1 (the prepare's invalid-point rows); the spread
    and gather-assemble kernels check every support against the face arrays
    before they touch it (an element whose box leaves the arrays takes the
    per-point path, and a point outside is skipped with AFSI_FLAG_INDEX), and
    any other reader of unconfirmed tables must do the same."""
    stencil: 'SharedAdaptiveStencil'
    x: torch.Tensor
    orders: torch.Tensor
    summary: torch.Tensor   # pinned host copy of the order summary and status word
    ready: torch.cuda.Event
    buffers: tuple = None
    status: torch.Tensor = None             # pinned copy of a table-free stencil's flags (note_transfers)
    status_ready: torch.cuda.Event = None


@dataclass(frozen=True)
class SharedAdaptiveStencil:
    base: torch.Tensor   # (2,T,3) int64: lattice 0 = faces, 1 = centres
    phi: torch.Tensor    # (2,T,3,4)
    rule: InteractionRule
    layout = 'shared'

    @property
    def storage_bytes(self):
        return self.base.numel() * self.base.element_size() + self.phi.numel() * self.phi.element_size()

    def expanded(self):
        """Per-component (3,T,3)/(3,T,3,4) tables (``mac/shared_stencil.py:13-19``)."""
        base = torch.stack([torch.stack([self.base[int(a != c), :, a] for a in range(3)], -1) for c in range(3)])
        phi = torch.stack([torch.stack([self.phi[int(a != c), :, a, :] for a in range(3)], 1) for c in range(3)])
        return base, phi


@dataclass(frozen=True)
class TableFreeStencil:
    """A rule without stencil tables: the positions ``x`` it was built for,
    the rule, and a device status word that the transfers OR their
    AFSI_FLAG_* bits into (checked by ``P2Transfer.confirm`` / ``check``)."""
    x: torch.Tensor
    rule: InteractionRule
    status: torch.Tensor
    layout = 'table-free'

    storage_bytes = 0


class P2Transfer:
    """Grid/quadrature state of the P2 CUDA transfer (no mass solve)."""

    nodes_per_cell = 10

    def __init__(self, grid, X, cells, *, point_density=2., max_order=8, max_points=12000000,
                 deterministic=False, transfer_dtype=None):
        if cells.dim() != 2 or cells.shape[1] != self.nodes_per_cell:
            raise ValueError(f'{type(self).__name__} requires {self.nodes_per_cell}-node tetrahedra')
        _lib.require_cuda(X)
        self.grid = grid
        self.node_count = X.shape[0]
        self.cells = cells.contiguous()
        cast = X.new_tensor
        self.origin, self.spacing = cast(grid.origin), cast(grid.spacing)
        self.limits = cast(grid.shape) - 2
        self.transfer_dtype = X.dtype if transfer_dtype is None else transfer_dtype
        if self.transfer_dtype != X.dtype and not (X.dtype == torch.float64 and self.transfer_dtype == torch.float32):
            raise ValueError('FP32 transfers are supported beside FP64 positions only')
        self.diagonal = torch.zeros((X.shape[0], 3), device=X.device, dtype=self.transfer_dtype)  # rhs template
        self._cast = None
        self.rules = RuleBuilder(X, self.cells, grid, point_density=point_density, max_order=max_order,
                                 max_points=max_points)
        self.deterministic = deterministic
        self._csr = None

    def rule(self, x):
        return self.rules(x)

    def prepare(self, x, *, buffers=None):
        """Rule + tables for positions ``x`` with one host read when the rule
        is unchanged: the order kernel and a prepare with the cached rule are
        queued together, then the order summary and the prepare's status word
        come back in one copy.  A changed rule discards the speculative tables
        and prepares again."""
        _lib.require_cuda(x)
        x = x.contiguous()
        last = self.rules.last
        orders, summary = self.rules.launch(x)
        speculative = None
        if last is not None:
            base, phi = _tables(x, last.point_count, buffers, self.transfer_dtype)
            _launch_prepare(self, x, last, base, phi, summary[-1:])
            speculative = base, phi
        counts = summary.cpu().tolist()
        rule = self.rules.finish(x, orders, counts)
        if speculative is not None and rule is last:
            _raise_flags(counts[-1])
            return SharedAdaptiveStencil(*speculative, rule)
        base, phi = prepare(self, x, rule, buffers=buffers)
        return SharedAdaptiveStencil(base, phi, rule)

    def prepare_deferred(self, x, *, buffers=None):
        """Rule + tables with no host read (rule selection without host syncs):
        the order kernel and a prepare with the cached rule are queued, and the
        order summary with the prepare's status word is copied to pinned host
        memory behind them.  The returned ``DeferredStencil.stencil`` is used
        at once; ``confirm`` checks it later, typically after the step's own
        host read, when the copy has long landed.  The first call has no
        cached rule and prepares synchronously (already confirmed)."""
        _lib.require_cuda(x)
        x = x.contiguous()
        last = self.rules.last
        if last is None:
            st = self.prepare(x, buffers=buffers)
            return DeferredStencil(st, x, None, None, None, buffers)
        orders, summary = self.rules.launch(x)
        base, phi = _tables(x, last.point_count, buffers, self.transfer_dtype)
        _launch_prepare(self, x, last, base, phi, summary[-1:])
        host = torch.empty(summary.shape, dtype=summary.dtype, pin_memory=True)
        host.copy_(summary, non_blocking=True)
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(x.device))
        return DeferredStencil(SharedAdaptiveStencil(base, phi, last), x, orders, host, ready, buffers)

    def prepare_table_free(self, x):
        """The rule for positions ``x`` and no tables, with no host read: as
        ``prepare_deferred``, the order kernel runs and its summary is copied
        to pinned memory behind it, and the cached rule is used at once.
        Returns a ``DeferredStencil`` whose ``stencil`` is a
        ``TableFreeStencil``; ``confirm`` settles the rule and raises the
        support / connectivity flags of the transfers that used it."""
        _lib.require_cuda(x)
        x = x.contiguous()
        last = self.rules.last
        if last is None:
            status = torch.zeros((), dtype=torch.int32, device=x.device)
            return DeferredStencil(TableFreeStencil(x, self.rules(x), status), x, None, None, None)
        orders, summary = self.rules.launch(x)
        status = summary[-1]  # the summary's spare slot, zeroed with it, takes the transfers' flags
        host = torch.empty(summary.shape, dtype=summary.dtype, pin_memory=True)
        host.copy_(summary, non_blocking=True)
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(x.device))
        return DeferredStencil(TableFreeStencil(x, last, status), x, orders, host, ready)

    def note_transfers(self, deferred):
        """After the transfers that use a deferred table-free stencil: copy its
        flag word to pinned memory behind them, so that ``confirm`` reads the
        copy (waiting for those transfers only) instead of the device word
        (which waits for everything queued on the stream since)."""
        if isinstance(deferred.stencil, TableFreeStencil):
            host = torch.empty((), dtype=torch.int32, pin_memory=True)
            host.copy_(deferred.stencil.status, non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(torch.cuda.current_stream(deferred.stencil.status.device))
            deferred.status, deferred.status_ready = host, ready

    def check(self, stencil):
        """Raise the flags a table-free stencil's transfers set (one host read)."""
        flags = int(stencil.status.item())
        if flags:
            stencil.status.zero_()
            _raise_flags(flags)

    def confirm(self, deferred):
        """Settle a deferred prepare: its stencil when the orders did not
        change (the common case; no work); a stencil prepared again,
        synchronously, with the new rule when they did (the caller redoes the
        transfers that used the old one); ``ValueError`` / ``RuntimeError``
        for a support or connectivity violation, as ``prepare`` raises them."""
        if isinstance(deferred.stencil, TableFreeStencil):
            st = deferred.stencil
            if deferred.summary is not None:
                deferred.ready.synchronize()
                counts = deferred.summary.tolist()
                rule = self.rules.finish(deferred.x, deferred.orders, counts)
                if rule is not st.rule:
                    return TableFreeStencil(st.x, rule, torch.zeros_like(st.status))
            if deferred.status is not None:
                deferred.status_ready.synchronize()
                flags = int(deferred.status.item())
                if flags:
                    st.status.zero_()
                    _raise_flags(flags)
            else:
                self.check(st)
            return st
        if deferred.summary is None:
            return deferred.stencil
        deferred.ready.synchronize()
        counts = deferred.summary.tolist()
        rule = self.rules.finish(deferred.x, deferred.orders, counts)
        if rule is deferred.stencil.rule:
            _raise_flags(counts[-1])
            return deferred.stencil
        base, phi = prepare(self, deferred.x, rule, buffers=deferred.buffers)
        return SharedAdaptiveStencil(base, phi, rule)

    def spread(self, coefficient, stencil):
        if self.deterministic:
            return spread_deterministic(self, coefficient, stencil)
        return spread(self, coefficient, stencil)

    def det_plan(self, stencil):
        """Tile-sorted rows of `stencil` for the deterministic spread (built once per stencil)."""
        key = (stencil.base.data_ptr(), stencil.base.shape[1], stencil.phi.dtype)
        if getattr(self, '_det', None) is not None and self._det[0] == key:
            return self._det[1]
        g = self.grid
        total = stencil.base.shape[1]
        code = dtype_code(stencil.phi.dtype)
        n = _lib.load().afsi_b200_det_plan_bytes(total, *g.shape, code)
        if n < 0:
            raise ValueError('stencil too large for the deterministic spread')
        plan = torch.empty(int(n), device=stencil.base.device, dtype=torch.uint8)
        word = _lib.status_word(plan.device)
        word.zero_()
        call('afsi_b200_det_plan', ptr(stencil.base), total, *g.shape, ptr(plan), plan.numel(), ptr(word), code,
             stream(plan.device))
        flags = int(word.item())
        if flags:
            word.zero_()
            raise RuntimeError('P2 stencil support outside the MAC face arrays')
        self._det = (key, plan)
        return plan

    def assemble_velocity(self, velocity, stencil):
        if self.deterministic:
            return assemble_velocity_deterministic(self, velocity, stencil)
        return assemble_velocity(self, velocity, stencil)

    def group_tables(self, rule):
        """(values N, weights W) of every group of `rule` in the transfer dtype
        (the rule's own tensors, or FP32 copies made once per rule)."""
        if self.transfer_dtype == rule.groups[0].weights.dtype:
            return [(g.values, g.weights) for g in rule.groups]
        if self._cast is None or self._cast[0] is not rule:
            self._cast = (rule, [(g.values.to(self.transfer_dtype).contiguous(),
                                  g.weights.to(self.transfer_dtype).contiguous()) for g in rule.groups])
        return self._cast[1]

    def node_csr(self, rule):
        """node -> (element*10+a) CSR over the rule's group order (built once per rule)."""
        if self._csr is not None and self._csr[0] is rule:
            return self._csr[1:]
        slots, offset = [], 0
        for g in rule.groups:
            slots.append(g.cells.reshape(-1))
        flat = torch.cat(slots)
        order = torch.argsort(flat, stable=True)
        counts = torch.bincount(flat, minlength=self.node_count)
        crow = torch.zeros(self.node_count + 1, dtype=torch.int64, device=flat.device)
        crow[1:] = torch.cumsum(counts, 0)
        self._csr = (rule, crow, order.contiguous())
        return crow, order


def _tables_ok(base, phi, total, x, dtype):
    return (base.shape == (2, total, 3) and phi.shape == (2, total, 3, 4) and base.dtype == torch.int64 and
            phi.dtype == dtype and base.device == x.device and phi.device == x.device and
            base.is_contiguous() and phi.is_contiguous())


def _tables(x, total, buffers, dtype=None):
    dtype = x.dtype if dtype is None else dtype
    if buffers is None:
        return (torch.empty((2, total, 3), device=x.device, dtype=torch.int64),
                torch.empty((2, total, 3, 4), device=x.device, dtype=dtype))
    base, phi = buffers
    if not _tables_ok(base, phi, total, x, dtype):
        raise ValueError('invalid P2 stencil buffers')
    return base, phi


def _launch_prepare(transfer, x, rule, base, phi, word):
    g = transfer.grid
    limits = [n - 2 for n in g.shape]
    offset = 0
    mixed = phi.dtype != x.dtype
    for group in rule.groups:
        if mixed:
            call('afsi_b200_fe_prepare_mixed', 10, ptr(x), x.shape[0], ptr(group.cells), group.cells.shape[0],
                 ptr(group.values), group.values.shape[0], _lib.doubles(g.origin), _lib.doubles(g.spacing),
                 _lib.doubles(limits), ptr(base), ptr(phi), rule.point_count, offset, ptr(word),
                 dtype_code(phi.dtype), stream(x.device))
        else:
            call('afsi_b200_p2_prepare', ptr(x), x.shape[0], ptr(group.cells), group.cells.shape[0],
                 ptr(group.values), group.values.shape[0], _lib.doubles(g.origin), _lib.doubles(g.spacing),
                 _lib.doubles(limits), ptr(base), ptr(phi), rule.point_count, offset, ptr(word),
                 dtype_code(x.dtype), stream(x.device))
        offset += group.weights.numel()


def _raise_flags(flags):
    if flags & _lib.FLAG_OVERFLOW:
        raise RuntimeError('an element support box exceeds the deterministic table-free spread\'s slot '
                           '(8 faces per axis); use the table form with deterministic=True')
    if flags & _lib.FLAG_TIMEOUT:
        raise RuntimeError('a P2 transfer gave up waiting for its staged stencil rows')
    if flags & _lib.FLAG_INDEX:
        raise RuntimeError('P2 connectivity outside the node range')
    if flags:
        raise ValueError('MAC IB support reaches a wall or is nonfinite; enlarge/refine the fluid box')


def prepare(transfer, x, rule, *, buffers=None):
    """``p2_cuda_transfer.prepare`` (``:18-39``): positions and shared tables
    of every group; ``ValueError`` when a point's support leaves the grid."""
    _lib.require_cuda(x)
    x = x.contiguous()
    base, phi = _tables(x, rule.point_count, buffers, getattr(transfer, 'transfer_dtype', x.dtype))
    word = _lib.status_word(x.device)
    word.zero_()
    _launch_prepare(transfer, x, rule, base, phi, word)
    flags = int(word.item())
    if flags:
        word.zero_()
        _raise_flags(flags)
    return base, phi


def spread(transfer, coefficient, stencil, *, events=None):
    """``p2_cuda_transfer.spread`` (``:42-49``): nodal coefficients -> MAC face
    fields, F_q = (N·coef)·W spread with weight/volume.  ``events`` (two CUDA
    events) bracket the native launches, excluding the output zero-fill."""
    _lib.require_cuda(coefficient)
    coefficient = coefficient.contiguous()
    if isinstance(stencil, TableFreeStencil):
        return _table_free_spread(transfer, coefficient, stencil, events)
    if coefficient.dtype != stencil.phi.dtype:
        raise ValueError('P2 spread coefficient dtype must match the stencil weights')
    g = transfer.grid
    fields = g.zeros(device=coefficient.device, dtype=coefficient.dtype)
    word = _lib.status_word(coefficient.device)
    offset = 0
    if events is not None:
        events[0].record()
    for group, (values, weights) in zip(stencil.rule.groups, _group_tables(transfer, stencil.rule)):
        call('afsi_b200_p2_spread', ptr(coefficient), coefficient.shape[0], ptr(group.cells), group.cells.shape[0],
             ptr(values), values.shape[0], ptr(weights), ptr(stencil.base), ptr(stencil.phi),
             stencil.base.shape[1], offset, *(ptr(f) for f in fields), *g.shape, float(g.volume), ptr(word),
             dtype_code(coefficient.dtype), stream(coefficient.device))
        offset += group.weights.numel()
    if events is not None:
        events[1].record()
    return fields


def _group_tables(transfer, rule):
    """Rule tables in the transfer's dtype (the reference's transfer objects
    have no precision form: their own tables)."""
    if hasattr(transfer, 'group_tables'):
        return transfer.group_tables(rule)
    return [(g.values, g.weights) for g in rule.groups]


def spread_deterministic(transfer, coefficient, stencil):
    """:func:`spread` without atomics and bitwise reproducible.  Tables: point
    forces (``afsi_b200_p2_point_forces``), then the tile-sorted deterministic
    spread (``afsi_b200_det_spread``) over the stencil's plan.  Table-free:
    element boxes in scratch slots reduced per face tile in a fixed order
    (``afsi_b200_fe_det_spread``)."""
    _lib.require_cuda(coefficient)
    coefficient = coefficient.contiguous()
    if isinstance(stencil, TableFreeStencil):
        return _table_free_spread(transfer, coefficient, stencil, deterministic=True)
    if coefficient.dtype != stencil.phi.dtype:
        raise ValueError('P2 spread coefficient dtype must match the stencil weights')
    g = transfer.grid
    total = stencil.base.shape[1]
    plan = transfer.det_plan(stencil)
    force = torch.empty((total, 3), device=coefficient.device, dtype=coefficient.dtype)
    word = _lib.status_word(coefficient.device)
    code = dtype_code(coefficient.dtype)
    s = stream(coefficient.device)
    offset = 0
    for group, (values, weights) in zip(stencil.rule.groups, _group_tables(transfer, stencil.rule)):
        call('afsi_b200_p2_point_forces', ptr(coefficient), coefficient.shape[0], ptr(group.cells),
             group.cells.shape[0], ptr(values), values.shape[0], ptr(weights), total, offset, float(g.volume),
             ptr(force), ptr(word), code, s)
        offset += group.weights.numel()
    fields = g.zeros(device=coefficient.device, dtype=coefficient.dtype)
    call('afsi_b200_det_spread', ptr(force), ptr(stencil.base), ptr(stencil.phi), total, *g.shape, ptr(plan),
         plan.numel(), *(ptr(f) for f in fields), code, s)
    return fields


def _velocity(transfer, velocity):
    transfer.grid.check_velocity(velocity)
    _lib.require_cuda(velocity[0])
    return tuple(v.contiguous() for v in velocity)


def assemble_velocity(transfer, velocity, stencil, *, events=None):
    """``p2_cuda_transfer.assemble_velocity`` (``:52-60``): MAC velocity ->
    nodal right-hand side rhs[a] = Σ_q N[q,a] W U(x_q).  ``events`` bracket
    the native launches."""
    velocity = _velocity(transfer, velocity)
    if isinstance(stencil, TableFreeStencil):
        return _table_free_assemble(transfer, velocity, stencil, events)
    if velocity[0].dtype != stencil.phi.dtype:
        raise ValueError('P2 velocity dtype must match the stencil weights')
    rhs = torch.zeros_like(transfer.diagonal)
    word = _lib.status_word(rhs.device)
    g = transfer.grid
    offset = 0
    if events is not None:
        events[0].record()
    for group, (values, weights) in zip(stencil.rule.groups, _group_tables(transfer, stencil.rule)):
        call('afsi_b200_p2_gather_assemble', *(ptr(v) for v in velocity), ptr(group.cells), group.cells.shape[0],
             ptr(values), values.shape[0], ptr(weights), ptr(stencil.base), ptr(stencil.phi),
             stencil.base.shape[1], offset, ptr(rhs), rhs.shape[0], *g.shape, ptr(word), dtype_code(rhs.dtype),
             stream(rhs.device))
        offset += group.weights.numel()
    if events is not None:
        events[1].record()
    return rhs


def assemble_velocity_deterministic(transfer, velocity, stencil):
    """Same result as :func:`assemble_velocity`, bitwise reproducible: element
    sums are written without atomics, then reduced per node in CSR order."""
    velocity = _velocity(transfer, velocity)
    if isinstance(stencil, TableFreeStencil):
        return _table_free_assemble(transfer, velocity, stencil, deterministic=True)
    rule = stencil.rule
    elements = sum(grp.cells.shape[0] for grp in rule.groups)
    local = torch.empty((elements, 10, 3), device=velocity[0].device, dtype=velocity[0].dtype)
    word = _lib.status_word(local.device)
    g = transfer.grid
    offset, first = 0, 0
    for group, (values, weights) in zip(rule.groups, _group_tables(transfer, rule)):
        call('afsi_b200_p2_gather_local', *(ptr(v) for v in velocity), ptr(group.cells), group.cells.shape[0],
             ptr(values), values.shape[0], ptr(weights), ptr(stencil.base), ptr(stencil.phi),
             stencil.base.shape[1], offset, local[first:].data_ptr(), *g.shape, ptr(word), dtype_code(local.dtype),
             stream(local.device))
        offset += group.weights.numel()
        first += group.cells.shape[0]
    crow, slot = transfer.node_csr(rule)
    rhs = torch.empty_like(transfer.diagonal)
    call('afsi_b200_node_reduce', ptr(local), elements * 10, ptr(crow), ptr(slot), rhs.shape[0], ptr(rhs), 0,
         ptr(word), dtype_code(rhs.dtype), stream(rhs.device))
    return rhs


# ------------------------------------------------------------ table-free form

def _geometry(transfer):
    """origin, spacing and support limits as ctypes arrays (made once per transfer)."""
    geo = getattr(transfer, '_geo', None)
    if geo is None:
        g = transfer.grid
        geo = _lib.doubles(g.origin), _lib.doubles(g.spacing), _lib.doubles([n - 2 for n in g.shape])
        transfer._geo = geo
    return geo


def _det_scratch(transfer, rule, dtype, device):
    """Scratch of the deterministic table-free spread for the largest group
    of `rule` (kept on the transfer and grown when needed)."""
    elements = max(grp.cells.shape[0] for grp in rule.groups)
    n = _lib.load().afsi_b200_fe_det_spread_bytes(elements, *transfer.grid.shape, dtype_code(dtype))
    if n < 0:
        raise ValueError('too many elements for the deterministic table-free spread')
    held = getattr(transfer, '_fe_det', None)
    if held is None or held.numel() < n or held.device != device:
        held = torch.empty(int(n), dtype=torch.uint8, device=device)
        transfer._fe_det = held
    return held


def _table_free_spread(transfer, coefficient, stencil, events=None, deterministic=False):
    """Spread with the rows formed in the kernel (``afsi_b200_fe_fused_spread``,
    or ``afsi_b200_fe_det_spread`` in the deterministic form)."""
    x = stencil.x
    if coefficient.dtype != transfer.transfer_dtype:
        raise ValueError('spread coefficient dtype must match the transfer dtype')
    g = transfer.grid
    fields = g.zeros(device=coefficient.device, dtype=coefficient.dtype)
    origin, spacing, limits = _geometry(transfer)
    scratch = _det_scratch(transfer, stencil.rule, coefficient.dtype, coefficient.device) if deterministic else None
    if events is not None:
        events[0].record()
    for group, (values, weights) in zip(stencil.rule.groups, _group_tables(transfer, stencil.rule)):
        args = (transfer.nodes_per_cell, ptr(x), x.shape[0], ptr(group.cells), group.cells.shape[0],
                ptr(group.values), ptr(values), values.shape[0], ptr(weights), ptr(coefficient), origin, spacing,
                limits, *(ptr(f) for f in fields), *g.shape, float(g.volume))
        tail = (ptr(stencil.status), dtype_code(x.dtype), dtype_code(coefficient.dtype), stream(coefficient.device))
        if deterministic:
            call('afsi_b200_fe_det_spread', *args, ptr(scratch), scratch.numel(), *tail)
        else:
            call('afsi_b200_fe_fused_spread', *args, *tail)
    if events is not None:
        events[1].record()
    return fields


def _table_free_assemble(transfer, velocity, stencil, events=None, deterministic=False):
    """Gather-assemble with the rows formed in the kernel (``afsi_b200_fe_fused_gather``;
    in the deterministic form element sums from ``afsi_b200_fe_fused_gather_local``
    reduced per node in CSR order)."""
    x = stencil.x
    if velocity[0].dtype != transfer.transfer_dtype:
        raise ValueError('velocity dtype must match the transfer dtype')
    if deterministic:
        return _table_free_assemble_local(transfer, velocity, stencil)
    rhs = torch.zeros_like(transfer.diagonal)
    origin, spacing, limits = _geometry(transfer)
    g = transfer.grid
    if events is not None:
        events[0].record()
    for group, (values, weights) in zip(stencil.rule.groups, _group_tables(transfer, stencil.rule)):
        call('afsi_b200_fe_fused_gather', transfer.nodes_per_cell, ptr(x), x.shape[0], ptr(group.cells),
             group.cells.shape[0], ptr(group.values), ptr(values), values.shape[0], ptr(weights),
             *(ptr(v) for v in velocity), origin, spacing, limits, ptr(rhs), *g.shape, ptr(stencil.status),
             dtype_code(x.dtype), dtype_code(rhs.dtype), stream(rhs.device))
    if events is not None:
        events[1].record()
    return rhs


def _table_free_assemble_local(transfer, velocity, stencil):
    rule = stencil.rule
    npc = transfer.nodes_per_cell
    elements = sum(grp.cells.shape[0] for grp in rule.groups)
    x = stencil.x
    local = torch.empty((elements, npc, 3), device=velocity[0].device, dtype=velocity[0].dtype)
    origin, spacing, limits = _geometry(transfer)
    g = transfer.grid
    first = 0
    for group, (values, weights) in zip(rule.groups, _group_tables(transfer, rule)):
        call('afsi_b200_fe_fused_gather_local', npc, ptr(x), x.shape[0], ptr(group.cells), group.cells.shape[0],
             ptr(group.values), ptr(values), values.shape[0], ptr(weights), *(ptr(v) for v in velocity), origin,
             spacing, limits, local[first:].data_ptr(), *g.shape, ptr(stencil.status), dtype_code(x.dtype),
             dtype_code(local.dtype), stream(local.device))
        first += group.cells.shape[0]
    crow, slot = transfer.node_csr(rule)
    rhs = torch.empty_like(transfer.diagonal)
    call('afsi_b200_node_reduce', ptr(local), elements * npc, ptr(crow), ptr(slot), rhs.shape[0], ptr(rhs), 0,
         ptr(stencil.status), dtype_code(rhs.dtype), stream(rhs.device))
    return rhs


class P1Transfer(P2Transfer):
    """Matrix-free P1 element transfer (the reference's ``AdaptiveP1Transfer``
    CUDA execution, ``mac/adaptive_cell.py:22-83`` -> ``mac/_triton_adaptive.py:
    25-128``, without the consistent-mass solve): the adaptive P1 rule
    (``mac/adaptive_transfer.py`` ``_orders``), then spread and gather-assemble
    of four-node elements with each point's position, bases and weights
    formed in the kernel; no stencil tables and no assembled operator.
    ``transfer_dtype=torch.float32`` beside FP64 positions keeps positions and
    bases in FP64 and runs the weights and transfers in FP32."""
    nodes_per_cell = 4

    def prepare(self, x, **_):
        """Rule for positions ``x`` (one host read when it changes); support and
        connectivity violations are raised by ``check`` / ``confirm``."""
        _lib.require_cuda(x)
        x = x.contiguous()
        return TableFreeStencil(x, self.rules(x), torch.zeros((), dtype=torch.int32, device=x.device))

    prepare_deferred = P2Transfer.prepare_table_free

    interpolate_rhs = P2Transfer.assemble_velocity
