"""Consistent-mass Jacobi-PCG on the B200.

Mirrors ``MassSolver`` / ``GraphMassSolver`` (``mac/mass_solver.py:39-103``,
``mac/mass_graph.py:129-225``): ``solve(rhs, initial=None)`` returns
``(x.clone(), SolveInfo(iterations, residual_norm, rhs_norm, tolerance))`` with
the reference's recurrence, breakdown guard, restart/check schedule,
true-residual acceptance and error messages.  The work runs in
``csrc/mass.cu``: the checks the reference makes on the host at every
``check_every`` iterations are made on the device, so a solve is one begin
launch plus one CUDA graph launch (a WHILE node over one iteration), and the
host reads the solver state once.  ``loop='host'`` keeps the reference's
blockwise host loop (one state read per check) over the same kernels.

CUDA only: there is no CPU path.
"""
import ctypes
from dataclasses import dataclass
from math import isfinite
import torch
from . import _lib

RUNNING, CONVERGED, BAD_INPUT, BREAKDOWN, NONFINITE, NOT_CONVERGED = range(6)
_SLOTS = 16
_RESIDUAL, _TOLERANCE, _BROKEN, _TRUE, _ITERATIONS, _STATUS, _RHS_NORM = 4, 5, 7, 9, 10, 11, 12


@dataclass(frozen=True)
class SolverOptions:
    """Same fields, defaults and validation as ``fluid/solvers.py:12-28``."""
    rtol: float = 1e-10
    atol: float = 1e-12
    max_iterations: int = 1000
    recompute_every: int = 40
    check_every: int = 1

    def __post_init__(self):
        if (not isfinite(self.rtol) or not isfinite(self.atol) or self.rtol < 0 or
                self.atol < 0 or self.rtol + self.atol == 0):
            raise ValueError('finite nonnegative tolerances, at least one positive, required')
        for name in ('max_iterations', 'recompute_every', 'check_every'):
            n = getattr(self, name)
            if not isinstance(n, int) or isinstance(n, bool) or n < 1:
                raise ValueError(f'{name} must be a positive integer')


@dataclass(frozen=True)
class SolveInfo:
    """Same fields as ``fluid/solvers.py:31-35``."""
    iterations: int
    residual_norm: float
    rhs_norm: float
    tolerance: float


def csr_arrays(mass, device):
    """(crow, col, values) of a CSR, COO or dense square matrix, int64 indices."""
    if mass.layout == torch.sparse_coo:
        mass = mass.coalesce().to_sparse_csr()
    elif mass.layout == torch.strided:
        mass = mass.to_sparse_csr()
    elif mass.layout != torch.sparse_csr:
        raise ValueError('mass matrix must be sparse CSR, sparse COO or dense')
    crow = mass.crow_indices().to(device=device, dtype=torch.int64).contiguous()
    col = mass.col_indices().to(device=device, dtype=torch.int64).contiguous()
    return crow, col, mass.values().to(device=device).contiguous()


class MassSolver:
    """Jacobi-PCG for the constant IB mass matrix (``mac/mass_solver.py:39-103``)."""

    def __init__(self, mass, diagonal, options=None, *, loop='graph'):
        if loop not in ('graph', 'host'):
            raise ValueError("mass solver loop must be 'graph' or 'host'")
        self.mass, self.diagonal = mass, diagonal
        self.options = options or SolverOptions()
        if not torch.isfinite(diagonal).all() or (diagonal <= 0).any():
            raise ValueError('Jacobi diagonal must be finite and positive')
        _lib.require_cuda(diagonal)
        if diagonal.ndim not in (1, 2) or (diagonal.ndim == 2 and not 1 <= diagonal.shape[1] <= 3):
            raise ValueError('mass solve needs a (nodes,) or (nodes, 1..3) diagonal')
        dtype_code = _lib.dtype_code(diagonal.dtype)
        rows = diagonal.shape[0]
        cols = 1 if diagonal.ndim == 1 else diagonal.shape[1]
        if mass.shape != (rows, rows):
            raise ValueError('mass matrix shape does not match the diagonal')
        self.loop = loop
        self.device = diagonal.device
        self.crow, self.col, self.values = csr_arrays(mass, self.device)
        if self.values.dtype != diagonal.dtype:
            raise ValueError('mass matrix and diagonal dtypes differ')
        self.x, self.r, self.d, self.Ad = [torch.empty_like(diagonal, memory_format=torch.contiguous_format)
                                           for _ in range(4)]
        # one value per row when the columns share it (the reference's expanded (nodes,) diagonal)
        per_row = diagonal.ndim == 1 or diagonal.stride(1) == 0 or bool((diagonal == diagonal[:, :1]).all())
        self._diag = (diagonal if diagonal.ndim == 1 else diagonal[:, 0]).contiguous().clone() if per_row else \
            diagonal.contiguous().clone()
        # 32-bit column indices halve the index traffic of every SpMV
        self._col32 = self.col.to(torch.int32) if rows < 2 ** 31 else None
        self._rhs = torch.empty_like(self.x)
        self._initial = torch.empty_like(self.x)
        self.state = torch.zeros(_SLOTS, dtype=torch.float64, device=self.device)
        self._scratch = torch.zeros(_lib.load().afsi_b200_pcg_scratch_bytes(), dtype=torch.uint8,
                                    device=self.device)
        self._host = torch.empty(_SLOTS, dtype=torch.float64, pin_memory=True)
        opt = self.options
        self.plan = _lib.PCGPlan(
            crow=self.crow.data_ptr(), col=None if self._col32 is not None else self.col.data_ptr(),
            col32=None if self._col32 is None else self._col32.data_ptr(), val=self.values.data_ptr(),
            diagonal=self._diag.data_ptr(), rhs=self._rhs.data_ptr(), initial=self._initial.data_ptr(),
            x=self.x.data_ptr(), r=self.r.data_ptr(), d=self.d.data_ptr(), Ad=self.Ad.data_ptr(),
            state=self.state.data_ptr(), scratch=self._scratch.data_ptr(), rows=rows, cols=cols, dtype=dtype_code,
            max_iterations=opt.max_iterations, check_every=opt.check_every, recompute_every=opt.recompute_every,
            diagonal_per_row=int(per_row), rtol=float(opt.rtol), atol=float(opt.atol))
        self._graph = None
        self.graph_body_launches = 0
        if loop == 'graph':
            handle = ctypes.c_void_p()
            before = _lib.launch_count()
            with torch.cuda.device(self.device):
                _lib.call('afsi_b200_pcg_graph_create', ctypes.byref(self.plan), ctypes.byref(handle))
            self._graph = handle.value
            self.graph_body_launches = _lib.launch_count() - before
            _lib.forget_launches(self.graph_body_launches)

    def __del__(self):
        graph, self._graph = getattr(self, '_graph', None), None
        if graph:
            try:
                _lib.call('afsi_b200_pcg_graph_destroy', graph)
            except Exception:
                pass

    def action(self, value, out):
        """out = M value (``MassSolver.action``), column by column through the CSR SpMV."""
        rows = self.crow.numel() - 1
        code = _lib.dtype_code(value.dtype)
        v = value.reshape(rows, -1)
        o = out.reshape(rows, -1)
        for c in range(v.shape[1]):
            _lib.call('afsi_b200_csr_spmv', _lib.ptr(self.crow), _lib.ptr(self.col), _lib.ptr(self.values), rows,
                      self.values.numel(), v[:, c:].data_ptr(), v.stride(0), o[:, c:].data_ptr(), o.stride(0), 1.0,
                      code, _lib.stream(self.device))

    def _read(self):
        self._host.copy_(self.state, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return self._host.tolist()

    @torch.no_grad()
    def solve(self, rhs, initial=None):
        opt = self.options
        for v in (rhs,) if initial is None else (rhs, initial):
            if v.shape != self.x.shape or v.dtype != self.x.dtype or v.device != self.x.device:
                raise ValueError('mass solve shape, dtype or device mismatch')
        self._rhs.copy_(rhs)
        if initial is None:
            self._initial.zero_()
        else:
            self._initial.copy_(initial)
        plan = ctypes.byref(self.plan)
        with torch.cuda.device(self.device):
            s = _lib.stream(self.device)
            _lib.call('afsi_b200_pcg_begin', plan, s)
            if self._graph is not None:
                _lib.call('afsi_b200_pcg_graph_launch', self._graph, s)
                state = self._read()
                # the WHILE body ran once per iteration (once, as no-ops, when begin stopped the solve)
                _lib.count_replay(self.graph_body_launches * max(int(state[_ITERATIONS]), 1))
            else:
                state = self._read()
                iteration = 0
                while state[_STATUS] == RUNNING and iteration < opt.max_iterations:
                    # blocks end where the reference checks (mac/mass_graph.py:202-205)
                    count = min(opt.check_every - iteration % opt.check_every,
                                opt.recompute_every - iteration % opt.recompute_every,
                                opt.max_iterations - iteration)
                    _lib.call('afsi_b200_pcg_iterations', plan, count, s)
                    iteration += count
                    state = self._read()
        return self._finish(state)

    def _finish(self, state):
        status = int(state[_STATUS])
        true_norm, tolerance = state[_TRUE], state[_TOLERANCE]
        if status == CONVERGED:
            return self.x.clone(), SolveInfo(int(state[_ITERATIONS]), true_norm, state[_RHS_NORM], tolerance)
        if status == BAD_INPUT:
            raise ValueError('finite mass RHS and initial guess required')
        if status == BREAKDOWN:
            raise RuntimeError('PCG breakdown: operator/preconditioner must be positive definite and finite')
        if status == NONFINITE:
            raise RuntimeError('nonfinite true PCG residual')
        if status == NOT_CONVERGED:
            raise RuntimeError(f'PCG did not converge: {true_norm:g} > {tolerance:g}')
        raise RuntimeError(f'mass solve stopped in state {status} after {int(state[_ITERATIONS])} iterations')


class GraphMassSolver(MassSolver):
    """``mac/mass_graph.py:129-225``: same results; the reference's option limits."""

    def __init__(self, mass, diagonal, options=None):
        super().__init__(mass, diagonal, options)
        if not 1 <= self.options.check_every <= 16 or self.options.recompute_every < 1:
            raise ValueError('graph PCG requires check_every in [1,16] and positive recompute_every')
