"""MAC geometric multigrid on the B200 kernels.

``GeometricMultigrid`` keeps the constructor and ``solve`` contract of
``afsi_torch/mac/multigrid.py:24-172`` (closed-box Neumann pressure, mean-zero
gauge) and ``ChannelMultigrid`` that of ``afsi_torch/mac2d/multigrid.py:16-134``
(inlet/outlet channel).  ``ChannelMultigrid(grid)`` with ``grid.periodic`` solves
the periodic-in-x / no-slip-in-y pressure problem, which has no reference
solver: same V-cycle, x-wrapped stencils, the mean-zero gauge and the rank-one
coarse inverse of the 3D solver.

``B200Kernels`` is the kernel object the reference workspaces call
(``smooth/residual/restrict/residual_restrict/prolong_add``,
``mac/_triton_mg.py:121-151``, ``mac2d/_triton_mg.py:78-100``).  Its ``smooth``
rebuilds the operator diagonal inside the kernel (the reference passes exactly
that diagonal), so no diagonal array is read.

The solve loop mirrors ``_solve_workspace``: start metrics (finiteness, mean,
norms) on the device with one host read, then blocks of ``check_every`` fused
V-cycles (optionally replayed as captured CUDA graphs) with one residual-norm
read per block.  Results are returned as fresh tensors, never workspace aliases.
"""
import ctypes
from dataclasses import dataclass
from math import isfinite, prod
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code


@dataclass(frozen=True)
class MGOptions:
    """``mac/multigrid.py:9-21``."""
    rtol: float = 1e-10
    atol: float = 1e-12
    max_cycles: int = 100
    smooth: int = 4
    check_every: int = 2

    def __post_init__(self):
        if (any(not isfinite(x) or x < 0 for x in (self.rtol, self.atol)) or
                self.rtol + self.atol == 0 or any(type(n) is not int or n < 1 for n in
                                                  (self.max_cycles, self.smooth, self.check_every))):
            raise ValueError('invalid multigrid options')


def _h2(spacing):
    return [h * h for h in spacing]


_BC_CODES = {'neumann': _lib.BC_NEUMANN, 'channel': _lib.BC_CHANNEL, 'periodic': _lib.BC_PERIODIC,
             'dirichlet': _lib.BC_DIRICHLET}


def _ih2(spacing):
    return [1 / h ** 2 for h in spacing]


class B200Kernels:
    """Kernel object for one boundary condition (3D closed or open box, 2D
    channel or periodic channel)."""

    def __init__(self, bc='neumann'):
        self.bc = _BC_CODES[bc]
        self.dim = 3 if bc in ('neumann', 'dirichlet') else 2
        self.name = 'b200' if bc == 'neumann' else f'b200-{bc}'

    def _shape(self, t):
        if t.dim() != self.dim:
            raise ValueError(f'expected a {self.dim}D pressure field')
        return _lib.int64s(list(t.shape) + [1] * (3 - self.dim))

    @staticmethod
    def _check(*ts):
        for t in ts:
            _lib.require_cuda(t)
            if not t.is_contiguous():
                raise ValueError('multigrid kernels need contiguous tensors')

    def smooth(self, p, rhs, diagonal, out, spacing):
        self._check(p, rhs, out)
        call('afsi_b200_mg_smooth', ptr(p), ptr(rhs), ptr(out), self._shape(p), _lib.doubles(_h2(spacing)),
             _lib.doubles(_ih2(spacing)), self.dim, self.bc, dtype_code(p.dtype), stream(p.device))

    def residual(self, p, rhs, out, spacing):
        self._check(p, rhs, out)
        call('afsi_b200_mg_residual', ptr(p), ptr(rhs), ptr(out), self._shape(p), _lib.doubles(_h2(spacing)),
             self.dim, self.bc, dtype_code(p.dtype), stream(p.device))

    def restrict(self, fine, out):
        self._check(fine, out)
        call('afsi_b200_mg_restrict', ptr(fine), ptr(out), self._shape(fine), self.dim, dtype_code(fine.dtype),
             stream(fine.device))

    def residual_restrict(self, p, rhs, out, spacing):
        self._check(p, rhs, out)
        call('afsi_b200_mg_residual_restrict', ptr(p), ptr(rhs), ptr(out), self._shape(p),
             _lib.doubles(_h2(spacing)), self.dim, self.bc, dtype_code(p.dtype), stream(p.device))

    def prolong_add(self, coarse, fine):
        self._check(coarse, fine)
        call('afsi_b200_mg_prolong_add', ptr(coarse), ptr(fine), self._shape(fine), self.dim, self.bc,
             dtype_code(fine.dtype), stream(fine.device))


def _levels(shape, spacing):
    """Coarsening rule of ``mac/multigrid.py:35-48``."""
    shapes, spacings = [], []
    shape, spacing = tuple(shape), tuple(spacing)
    while True:
        shapes.append(shape)
        spacings.append(spacing)
        if min(shape) <= 4 or any(n % 2 for n in shape):
            break
        shape = tuple(n // 2 for n in shape)
        spacing = tuple(2 * h for h in spacing)
    if prod(shape) > 512:
        raise ValueError('MAC dimensions must coarsen to <=512 cells; use powers of two')
    return shapes, spacings


def _coarse_matrix(shape, spacing, bc):
    """Dense coarsest operator (float64, CPU): -Δ with the level's BC, plus
    11ᵀ/n when singular (``mac/multigrid.py:49-59``, ``mac2d/multigrid.py:41-45``,
    ``mac/dirichlet_mg.py:30-34``)."""
    n = prod(shape)
    ids = torch.arange(n).reshape(shape)
    A = torch.zeros((n, n), dtype=torch.float64)
    dim = len(shape)
    for c, h in enumerate(spacing):
        w = 1 / h ** 2
        if bc == 'periodic' and c == 0:
            a = ids.reshape(-1)
            b = torch.roll(ids, -1, 0).reshape(-1)
        else:
            sl_a = [slice(None)] * dim
            sl_b = [slice(None)] * dim
            sl_a[c] = slice(None, -1)
            sl_b[c] = slice(1, None)
            a, b = ids[tuple(sl_a)].reshape(-1), ids[tuple(sl_b)].reshape(-1)
        for row, col, val in ((a, a, w), (b, b, w), (a, b, -w), (b, a, -w)):
            A.index_put_((row, col), torch.full(row.shape, val, dtype=torch.float64), accumulate=True)
    if bc == 'channel':
        last = ids[-1].reshape(-1)
        A.index_put_((last, last), torch.full(last.shape, 2 / spacing[0] ** 2, dtype=torch.float64),
                     accumulate=True)
    elif bc == 'dirichlet':
        # zero pressure half a cell outside every face (mac/open_boundary.py:14-24)
        for c, h in enumerate(spacing):
            for end in (0, -1):
                face = ids.select(c, end).reshape(-1)
                A.index_put_((face, face), torch.full(face.shape, 2 / h ** 2, dtype=torch.float64),
                             accumulate=True)
    else:
        A += 1. / n
    return A


class _Workspace:
    """Fixed-address level buffers, reduction scratch and the native plan."""

    def __init__(self, shapes, spacings, bc, dtype, device, smooth, coarse_dtype):
        self.p = [torch.zeros(s, device=device, dtype=dtype) for s in shapes]
        self.ping = [torch.zeros(s, device=device, dtype=dtype) for s in shapes]
        self.rhs = [torch.zeros(s, device=device, dtype=dtype) for s in shapes]
        bcode = _BC_CODES[bc]
        plan = _lib.MGPlan()
        plan.dim = len(shapes[0])
        plan.bc = bcode
        plan.levels = len(shapes)
        plan.smooth = smooth
        plan.dtype = dtype_code(dtype)
        plan.coarse_dtype = dtype_code(coarse_dtype)
        for l, (s, h) in enumerate(zip(shapes, spacings)):
            L = plan.level[l]
            dims = list(s) + [1] * (3 - len(s))
            hh = list(h) + [1.] * (3 - len(h))
            for a in range(3):
                L.shape[a] = dims[a]
                L.h2[a] = hh[a] * hh[a]
                L.inv_h2[a] = 1 / hh[a] ** 2
            L.p, L.ping, L.rhs = ptr(self.p[l]), ptr(self.ping[l]), ptr(self.rhs[l])
        nbytes = _lib.load().afsi_b200_mg_scratch_bytes(ctypes.byref(plan))
        self.scratch = torch.zeros(int(nbytes), device=device, dtype=torch.uint8)
        plan.scratch = ptr(self.scratch)
        self.plan = plan
        self.sync = torch.zeros(int(_lib.load().afsi_b200_mg_sync_bytes()), device=device, dtype=torch.uint8)
        self.info = torch.zeros(3, device=device, dtype=torch.float64)
        self.stats = torch.zeros(12, device=device, dtype=torch.float64)
        self.norm = torch.zeros(1, device=device, dtype=torch.float64)
        self.stat_scratch = torch.zeros(4096 * 8 * 4 + 64, device=device, dtype=torch.uint8)
        self.allocated_bytes = sum(t.numel() * t.element_size()
                                   for group in (self.p, self.ping, self.rhs) for t in group)

    def set_coarse(self, inverse):
        self.coarse_inverse = inverse
        self.plan.coarse_inverse = ptr(inverse)

    def vcycles(self, count):
        call('afsi_b200_mg_vcycles', ctypes.byref(self.plan), count, stream(self.p[0].device))

    def persistent(self, cycles, *, tol=None, check_every=1):
        """`cycles` V-cycles in one cooperative launch; with `tol`, stop on the
        device once the residual norm is <= tol (checked every `check_every`)."""
        call('afsi_b200_mg_persistent', ctypes.byref(self.plan), int(cycles), 0 if tol is None else 1,
             int(check_every), 0. if tol is None else float(tol), ptr(self.info), ptr(self.sync),
             stream(self.p[0].device))

    def residual_norm(self):
        call('afsi_b200_mg_residual_norm', ctypes.byref(self.plan), ptr(self.norm), stream(self.p[0].device))
        return self.norm[0]

    def vector_stats(self, x, out):
        call('afsi_b200_vector_stats', ptr(x), x.numel(), ptr(out), ptr(self.stat_scratch), dtype_code(x.dtype),
             stream(x.device))

    def subtract_mean(self, x, stats):
        call('afsi_b200_subtract_mean', ptr(x), x.numel(), ptr(stats), dtype_code(x.dtype), stream(x.device))


class _Solver:
    bc = 'neumann'
    # reference messages (mac/multigrid.py:125-172, mac2d/multigrid.py:85-111)
    _bad_rhs = 'invalid pressure RHS'
    _bad_initial = 'invalid initial pressure'
    _nonfinite_input = 'finite pressure RHS/initial guess required'
    _nonfinite_residual = 'nonfinite multigrid residual'
    _not_converged = 'pressure multigrid did not converge'

    def __init__(self, grid, *, device='cuda', dtype=torch.float64, options=None, backend='b200-graph',
                 coarse_dtype=None, smoother='jacobi'):
        if backend not in ('b200', 'b200-graph', 'b200-persistent'):
            raise ValueError('pressure backend must be b200, b200-graph or b200-persistent')
        if smoother not in ('jacobi', 'red-black'):
            raise ValueError("smoother must be 'jacobi' (the reference's) or 'red-black'")
        if smoother == 'red-black' and backend == 'b200-persistent':
            raise ValueError('the persistent backend runs the Jacobi smoother only')
        self.smoother = smoother
        device = torch.device(device)
        if device.type != 'cuda':
            raise ValueError('the B200 multigrid requires a CUDA device; there is no CPU fallback')
        _lib.load()
        self.options = MGOptions() if options is None else options
        self.grid = grid
        self.shapes, self.spacings = _levels(grid.shape, grid.spacing)
        self.dtype = dtype
        self.coarse_dtype = dtype if coarse_dtype is None else coarse_dtype
        A = _coarse_matrix(self.shapes[-1], self.spacings[-1], self.bc)
        self.coarse_inverse = torch.linalg.inv(A).to(device=device, dtype=self.coarse_dtype)
        self.kernels = B200Kernels(self.bc)
        self.workspace = _Workspace(self.shapes, self.spacings, self.bc, dtype, device, self.options.smooth,
                                    self.coarse_dtype)
        self.workspace.set_coarse(self.coarse_inverse)
        self.workspace.plan.smoother = 1 if smoother == 'red-black' else 0
        self.backend = self.kernels.name + {'b200': '', 'b200-graph': '-graph', 'b200-persistent': '-persistent'}[backend]
        if smoother == 'red-black':
            self.backend += '-red-black'
        self.persistent = backend == 'b200-persistent'
        self.graphs = {}
        if backend == 'b200-graph':
            self._capture()

    @property
    def singular(self):
        return self.bc in ('neumann', 'periodic')

    # -- execution
    def _capture(self):
        w = self.workspace
        device = w.p[0].device
        with torch.cuda.device(device):
            s = torch.cuda.Stream(device=device)
            s.wait_stream(torch.cuda.current_stream(device))
            with torch.cuda.stream(s):
                for _ in range(2):
                    w.vcycles(self.options.check_every)
            torch.cuda.current_stream(device).wait_stream(s)
            self.graph_launches = {}
            for count in range(1, self.options.check_every + 1):
                g = torch.cuda.CUDAGraph()
                before = _lib.launch_count()
                with torch.cuda.graph(g, stream=s):
                    w.vcycles(count)
                self.graph_launches[count] = _lib.launch_count() - before
                _lib.forget_launches(self.graph_launches[count])
                self.graphs[count] = g
            torch.cuda.current_stream(device).wait_stream(s)
            for t in (*w.p, *w.ping, *w.rhs):
                t.zero_()
        self._capture_loop()

    def _capture_loop(self):
        """The host solve loop as one device graph (``afsi_b200_mg_solve_graph_create``):
        blocks of ``check_every`` V-cycles with the residual check between them."""
        w = self.workspace
        self.loop_graph = None
        if self.options.max_cycles < self.options.check_every:
            return
        self.loop = torch.zeros(4, dtype=torch.float64, device=w.p[0].device)
        handle = ctypes.c_void_p()
        before = _lib.launch_count()
        with torch.cuda.device(w.p[0].device):
            _lib.call('afsi_b200_mg_solve_graph_create', ctypes.byref(w.plan), self.options.check_every,
                      self.options.max_cycles, _lib.ptr(self.loop), _lib.ptr(w.norm), ctypes.byref(handle))
        self.loop_graph = handle.value
        self.loop_body_launches = _lib.launch_count() - before
        _lib.forget_launches(self.loop_body_launches)
        # the same loop with the solve's start in front of it: one launch and one host read per solve
        self.params = torch.zeros(4, dtype=torch.float64, device=w.p[0].device)
        self._params_key = None
        self._generation = 0
        handle = ctypes.c_void_p()
        before = _lib.launch_count()
        with torch.cuda.device(w.p[0].device):
            _lib.call('afsi_b200_mg_solve_graph_create_started', ctypes.byref(w.plan), self.options.check_every,
                      self.options.max_cycles, _lib.ptr(self.loop), _lib.ptr(w.norm), _lib.ptr(w.stats),
                      _lib.ptr(w.stat_scratch), _lib.ptr(self.params), ctypes.byref(handle))
        self.started_graph = handle.value
        captured = _lib.launch_count() - before
        _lib.forget_launches(captured)
        self.start_launches = captured - self.loop_body_launches

    def __del__(self):
        for name in ('loop_graph', 'started_graph'):
            graph = getattr(self, name, None)
            if graph:
                try:
                    _lib.call('afsi_b200_mg_solve_graph_destroy', graph)
                except Exception:
                    pass
                setattr(self, name, None)

    def _run_loop(self, tol):
        """Device-side check loop from cycle 0; returns (cycles, residual)."""
        lp = self.loop
        lp.zero_()
        lp[0].fill_(tol)
        _lib.call('afsi_b200_mg_solve_graph_launch', self.loop_graph, _lib.stream(lp.device))
        _, cycles, residual, nonfinite = lp.tolist()
        cycles = int(cycles)
        _lib.count_replay(cycles // self.options.check_every * self.loop_body_launches)
        if nonfinite:
            raise RuntimeError(self._nonfinite_residual)
        return cycles, residual

    def advance(self, count):
        if self.persistent:
            self.workspace.persistent(count)
            return self.workspace.p[0]
        if self.graphs:
            self.graphs[count].replay()
            _lib.count_replay(self.graph_launches[count])
        else:
            self.workspace.vcycles(count)
        return self.workspace.p[0]

    def cycle(self):
        """One V-cycle on the workspace iterate (for parity checks)."""
        self.workspace.vcycles(1)
        return self.workspace.p[0]

    def initialize(self, p, rhs):
        self.workspace.p[0].copy_(p)
        self.workspace.rhs[0].copy_(rhs)

    def residual_norm(self):
        return self.workspace.residual_norm()

    # -- solve
    def _start(self, rhs, initial):
        """Copy in, gauge-shift (singular BCs) and measure; one host read.

        Returns raw-rhs (sum, sum|x|, finite), p finite, ||rhs|| after the
        shift and the initial residual norm (``_start_metrics``,
        ``mac/multigrid.py:68-73``)."""
        w = self.workspace
        w.rhs[0].copy_(rhs)
        w.p[0].zero_() if initial is None else w.p[0].copy_(initial)
        st = w.stats
        w.vector_stats(w.rhs[0], st[0:4])
        w.vector_stats(w.p[0], st[4:8])
        if self.singular:
            w.subtract_mean(w.rhs[0], st[0:4])
            w.subtract_mean(w.p[0], st[4:8])
            w.vector_stats(w.rhs[0], st[8:12])
        else:
            st[8:12].copy_(st[0:4])
        w.residual_norm()
        v = torch.cat((st, w.norm)).tolist()
        return dict(rhs_sum=v[0], rhs_abs=v[1], rhs_finite=v[3], p_finite=v[7], rhs_sq=v[10], residual=v[12])

    def _launch_started(self, rhs, initial, rtol, rel, n):
        """Copy in and launch the started loop graph
        (``afsi_b200_mg_solve_graph_create_started``: start and check loop on
        the device); returns the device snapshot of the statistics, the initial
        norm and the loop state, to be read by ``_read_started``."""
        w = self.workspace
        w.rhs[0].copy_(rhs)
        w.p[0].zero_() if initial is None else w.p[0].copy_(initial)
        key = (float(rtol), float(self.options.atol), rel, float(n))
        if key != self._params_key:
            self.params.copy_(torch.tensor(key, dtype=torch.float64))
            self._params_key = key
        _lib.call('afsi_b200_mg_solve_graph_launch', self.started_graph, _lib.stream(w.p[0].device))
        self._generation += 1
        return torch.cat((w.stats, w.norm, self.loop))

    def _read_started(self, snapshot):
        """One host read of a started solve: the start metrics of ``_start``,
        the tolerance, the cycles run, the last residual norm and the loop's
        nonfinite flag."""
        v = snapshot.tolist()
        tol, cycles, residual, nonfinite = v[13], int(v[14]), v[15], v[16]
        _lib.count_replay(self.start_launches + cycles // self.options.check_every * self.loop_body_launches)
        m = dict(rhs_sum=v[0], rhs_abs=v[1], rhs_finite=v[3], p_finite=v[7], rhs_sq=v[10], residual=v[12])
        return m, tol, cycles, residual, nonfinite

    def _solve_args(self, rhs, initial, rtol):
        rtol = self.options.rtol if rtol is None else rtol
        if not isfinite(rtol) or rtol < 0:
            raise ValueError('invalid multigrid solve tolerance')
        if rhs.shape != self.shapes[0] or rhs.device != self.workspace.p[0].device or rhs.dtype != self.dtype:
            raise ValueError(self._bad_rhs)
        if initial is not None and (initial.shape != rhs.shape or initial.device != rhs.device
                                    or initial.dtype != rhs.dtype):
            raise ValueError(self._bad_initial)
        return rtol

    def _started(self):
        return getattr(self, 'started_graph', None) and not self.persistent

    def solve(self, rhs, initial=None, *, rtol=None):
        rtol = self._solve_args(rhs, initial, rtol)
        if self._started():
            n = rhs.numel()
            rel = 1e-10 if self.dtype == torch.float64 else 1e-6
            snapshot = self._launch_started(rhs, initial, rtol, rel, n)
            return self._solve_now(rhs, initial, rtol, self._read_started(snapshot))
        return self._solve_now(rhs, initial, rtol, None)

    def solve_deferred(self, rhs, initial=None, *, rtol=None):
        """``solve`` in two halves: the device work is launched now and the
        returned ``PendingSolve``'s ``result()`` makes the host read, the input
        checks and any host tail later, so that a caller can queue further
        work first.  With the started loop graph the solution is copied out at
        launch time; other backends solve at once."""
        rtol = self._solve_args(rhs, initial, rtol)
        if self._started():
            n = rhs.numel()
            rel = 1e-10 if self.dtype == torch.float64 else 1e-6
            snapshot = self._launch_started(rhs, initial, rtol, rel, n)
            return PendingSolve(self, snapshot, self.workspace.p[0].clone(), rhs, initial, rtol, self._generation)
        return PendingSolve.done(self._solve_now(rhs, initial, rtol, None))

    def _solve_now(self, rhs, initial, rtol, started):
        """The host half of a solve (``mac/multigrid.py:125-172``); `started`
        is the result of ``_read_started`` for a launched started graph, else
        the start runs here."""
        w = self.workspace
        n = rhs.numel()
        rel = 1e-10 if self.dtype == torch.float64 else 1e-6
        if started is not None:
            m, tol, cycle, loop_residual, nonfinite = started
        else:
            m = self._start(rhs, initial)
        if self.singular:
            if not m['rhs_finite']:
                raise ValueError('invalid pressure RHS')
            # the reference's screen in FP64; an FP32 right-hand side that was
            # mean-free before rounding keeps a mean of its rounding errors
            if abs(m['rhs_sum'] / n) > 1e-12 + rel * (m['rhs_abs'] / n):
                raise ValueError('incompatible Neumann pressure RHS: net flux must vanish')
            if not m['p_finite']:
                raise ValueError('invalid initial pressure')
        elif not (m['rhs_finite'] and m['p_finite']):
            raise ValueError(self._nonfinite_input)
        rhs_norm, residual = m['rhs_sq'] ** .5, m['residual']
        if not isfinite(rhs_norm) or not isfinite(residual):
            if self.bc == 'dirichlet':
                raise ValueError(self._nonfinite_input)
            raise RuntimeError('nonfinite multigrid residual or RHS norm')
        if started is not None:
            if nonfinite:
                raise RuntimeError(self._nonfinite_residual)
            residual = loop_residual
        else:
            tol = max(self.options.atol, rtol * rhs_norm)
            cycle = 0
        if self.persistent and residual > tol:
            # whole loop on the device: same check schedule, one host read
            w.persistent(self.options.max_cycles, tol=tol, check_every=self.options.check_every)
            cycle, residual, failed = w.info.tolist()
            cycle = int(cycle)
            if failed:
                raise RuntimeError('persistent multigrid barrier timed out')
            if not isfinite(residual):
                raise RuntimeError('nonfinite multigrid residual')
        if started is None and getattr(self, 'loop_graph', None) and residual > tol:
            cycle, residual = self._run_loop(tol)
        while residual > tol and cycle < self.options.max_cycles:
            count = min(self.options.check_every, self.options.max_cycles - cycle)
            self.advance(count)
            cycle += count
            residual = self.residual_norm().item()
            if not isfinite(residual):
                raise RuntimeError(self._nonfinite_residual)
        if residual > tol:
            raise RuntimeError(f'{self._not_converged}: {residual:g} > {tol:g}')
        return w.p[0].clone(), dict(cycles=cycle, residual_norm=residual, tolerance=tol, backend=self.backend)


class PendingSolve:
    """The host half of a multigrid solve launched by ``solve_deferred``:
    ``result()`` reads the device state once, makes the reference's input
    checks (raising as ``solve`` does) and returns (p, info).  A solve that
    needs host cycles after the device loop (the loop stopped short of
    max_cycles) runs them on the solver's workspace while no later solve has
    been launched on it, else solves again from a copy of its inputs."""

    def __init__(self, solver, snapshot, p, rhs, initial, rtol, generation):
        self.solver, self.snapshot, self.p, self.rtol, self.generation = solver, snapshot, p, rtol, generation
        self.rhs = rhs.clone()
        self.initial = None if initial is None else initial.clone()
        self._done = None

    @classmethod
    def done(cls, outcome):
        pending = cls.__new__(cls)
        pending._done = outcome
        pending.p = outcome[0]
        return pending

    def result(self):
        if self._done is None:
            s = self.solver
            started = s._read_started(self.snapshot)
            m, tol, cycles, residual, nonfinite = started
            needs_host = (residual > tol and cycles < s.options.max_cycles and not nonfinite and isfinite(residual)
                          and m['rhs_finite'] and m['p_finite'])
            if needs_host and s._generation != self.generation:
                # the workspace holds a later solve: solve this one again
                self._done = s.solve(self.rhs, self.initial, rtol=self.rtol)
            else:
                p, info = s._solve_now(self.rhs, self.initial, self.rtol, started)
                self._done = (p if needs_host else self.p), info
        return self._done


class GeometricMultigrid(_Solver):
    """Closed-box 3D pressure V-cycle solver (``mac/multigrid.py:24-172``)."""
    bc = 'neumann'


class DirichletMultigrid(_Solver):
    """Open-box 3D pressure solver, zero pressure on the physical faces
    (``mac/dirichlet_mg.py:10-123``): same V-cycle with the face ghost -p, odd
    extension in the prolongation, no gauge.  ``backend`` also accepts the
    reference's names ('torch', 'fused', 'workspace' run per-block launches,
    'graph' the captured solve graph)."""
    bc = 'dirichlet'
    _bad_rhs = 'Dirichlet pressure RHS shape/dtype/device mismatch'
    _bad_initial = 'invalid initial Dirichlet pressure'
    _nonfinite_input = 'nonfinite Dirichlet pressure input'
    _nonfinite_residual = 'nonfinite Dirichlet multigrid residual'
    _not_converged = 'Dirichlet multigrid failed'

    def __init__(self, grid, *, backend='b200-graph', **kwargs):
        backend = {'torch': 'b200', 'fused': 'b200', 'workspace': 'b200', 'graph': 'b200-graph'}.get(backend, backend)
        super().__init__(grid, backend=backend, **kwargs)


class ChannelMultigrid(_Solver):
    """2D channel (``mac2d/multigrid.py:16-134``) or, with ``grid.periodic``,
    the periodic-x / Neumann-y problem."""

    def __init__(self, grid, **kwargs):
        self.bc = 'periodic' if getattr(grid, 'periodic', False) else 'channel'
        super().__init__(grid, **kwargs)


class RefinedMultigrid:
    """Precision form of the pressure solve: FP32 V-cycles inside FP64
    iterative refinement.

    No counterpart in the reference, whose solvers are FP64 throughout
    (``mac/multigrid.py:125-172``).  The iterate, the right-hand side, every
    residual and the dense coarsest solve stay FP64; each refinement forms the
    FP64 residual r = rhs - A p (``afsi_b200_mg_refine_residual``, the
    reference operator), hands it to FP32 V-cycles as float, runs them until
    the FP32 residual falls by ``inner_rtol`` (the device-side solve loop of
    the FP32 solver) and adds the correction to p in FP64
    (``afsi_b200_mg_refine_correct``).  It stops when the FP64 residual meets
    ``max(atol, rtol ||rhs||)``, the FP64 solver's tolerance; the method differs
    from the FP64 solver's (another cycle count), so results agree at the solve
    tolerance, not bitwise.  Singular problems (Neumann, periodic) keep the
    mean-zero gauge: the right-hand side and initial guess are shifted as in the
    FP64 solver, each FP32 residual is shifted before its V-cycles, and the
    final iterate is shifted once more in FP64.
    """

    def __init__(self, grid, *, bc=None, device='cuda', options=None, inner_rtol=1e-5, inner_cycles=40,
                 max_refinements=8, backend='b200-graph', smoother='jacobi'):
        self.options = MGOptions() if options is None else options
        if not 0 < inner_rtol < 1 or max_refinements < 1:
            raise ValueError('refinement needs 0 < inner_rtol < 1 and max_refinements >= 1')
        kind = bc or ('periodic' if getattr(grid, 'periodic', False) else
                      'channel' if len(grid.shape) == 2 else 'neumann')
        cls = {'neumann': GeometricMultigrid, 'dirichlet': DirichletMultigrid, 'channel': ChannelMultigrid,
               'periodic': ChannelMultigrid}[kind]
        inner_opts = MGOptions(rtol=inner_rtol, atol=0., max_cycles=inner_cycles, smooth=self.options.smooth,
                               check_every=self.options.check_every)
        self.inner = cls(grid, device=device, dtype=torch.float32, coarse_dtype=torch.float64, options=inner_opts,
                         backend=backend, smoother=smoother)
        self.bc = self.inner.bc
        self.inner_rtol = inner_rtol
        self.max_refinements = max_refinements
        w = self.inner.workspace
        self.shape = tuple(self.inner.shapes[0])
        dev = w.p[0].device
        self.p = torch.zeros(self.shape, device=dev, dtype=torch.float64)
        self.rhs = torch.zeros_like(self.p)
        self.stats = torch.zeros(8, device=dev, dtype=torch.float64)
        self.norm = torch.zeros(1, device=dev, dtype=torch.float64)
        self._shape = _lib.int64s(self.shape)
        h = self.inner.spacings[0]
        self._h2 = _lib.doubles([x * x for x in h])
        self._dim = len(self.shape)
        nbytes = _lib.load().afsi_b200_mg_refine_scratch_bytes(self._shape, self._dim, _BC_CODES[self.bc])
        if nbytes < 0:
            raise ValueError('grid not supported by the refinement kernels')
        self.scratch = torch.zeros(int(nbytes), device=dev, dtype=torch.uint8)
        self.backend = self.inner.backend + '-refined'

    @property
    def singular(self):
        return self.bc in ('neumann', 'periodic')

    def _residual(self):
        """FP64 residual of self.p into the FP32 solver's rhs; its norm (one host read)."""
        w = self.inner.workspace
        call('afsi_b200_mg_refine_residual', ptr(self.p), ptr(self.rhs), ptr(w.rhs[0]), self._shape, self._h2,
             self._dim, _BC_CODES[self.bc], ptr(self.norm), ptr(self.scratch), stream(self.p.device))
        return self.norm.item()

    def _inner_solve(self, norm):
        """FP32 V-cycles on the residual from a zero start; returns the cycles run."""
        inner, w = self.inner, self.inner.workspace
        if self.singular:
            w.vector_stats(w.rhs[0], w.stats[0:4])
            w.subtract_mean(w.rhs[0], w.stats[0:4])
        w.p[0].zero_()
        tol = self.inner_rtol * norm
        if getattr(inner, 'loop_graph', None):
            cycles, residual = inner._run_loop(tol)
        else:
            cycles, residual = 0, float('inf')
            while residual > tol and cycles + inner.options.check_every <= inner.options.max_cycles:
                inner.advance(inner.options.check_every)
                cycles += inner.options.check_every
                residual = inner.residual_norm().item()
        if not isfinite(residual):
            raise RuntimeError('nonfinite multigrid residual in the FP32 correction')
        call('afsi_b200_mg_refine_correct', ptr(self.p), ptr(w.p[0]), self.p.numel(), stream(self.p.device))
        return cycles

    @torch.no_grad()
    def solve(self, rhs, initial=None, *, rtol=None):
        rtol = self.options.rtol if rtol is None else rtol
        if not isfinite(rtol) or rtol < 0:
            raise ValueError('invalid multigrid solve tolerance')
        if rhs.shape != self.shape or rhs.dtype != torch.float64 or rhs.device != self.p.device:
            raise ValueError('refined pressure solve needs an FP64 right-hand side on the solver device')
        if initial is not None and (initial.shape != self.shape or initial.dtype != torch.float64
                                    or initial.device != self.p.device):
            raise ValueError('invalid initial pressure')
        w = self.inner.workspace
        self.rhs.copy_(rhs)
        self.p.zero_() if initial is None else self.p.copy_(initial)
        w.vector_stats(self.rhs, self.stats[0:4])
        w.vector_stats(self.p, self.stats[4:8])
        raw = self.stats.tolist()
        n = rhs.numel()
        if not (raw[3] and raw[7]):
            raise ValueError('finite pressure RHS/initial guess required')
        if self.singular:
            if abs(raw[0] / n) > 1e-12 + 1e-10 * (raw[1] / n):
                raise ValueError('incompatible Neumann pressure RHS: net flux must vanish')
            w.subtract_mean(self.rhs, self.stats[0:4])
            w.subtract_mean(self.p, self.stats[4:8])
            w.vector_stats(self.rhs, self.stats[0:4])
        rhs_norm = self.stats[2].item() ** .5
        tol = max(self.options.atol, rtol * rhs_norm)
        cycles = refinements = 0
        residual = self._residual()
        while residual > tol and refinements < self.max_refinements and isfinite(residual):
            cycles += self._inner_solve(residual)
            refinements += 1
            residual = self._residual()
        if not isfinite(residual):
            raise RuntimeError('nonfinite multigrid residual')
        if residual > tol:
            raise RuntimeError(f'refined pressure multigrid did not converge: {residual:g} > {tol:g}')
        if self.singular:
            w.vector_stats(self.p, self.stats[4:8])
            w.subtract_mean(self.p, self.stats[4:8])
        return self.p.clone(), dict(cycles=cycles, refinements=refinements, residual_norm=residual, tolerance=tol,
                                    backend=self.backend)
