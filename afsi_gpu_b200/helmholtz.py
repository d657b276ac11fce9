"""CN Helmholtz Jacobi sweeps and Stokes residual reductions on the B200.

``HelmholtzKernels`` is the kernel object of ``mac/helmholtz.py``'s
``HelmholtzWorkspace`` (the reference builds ``_triton_helmholtz.HelmholtzKernels``,
``mac/helmholtz.py:44-47``): ``initialize(b, p, diagonal, rhs, u, parameters,
grid)`` and ``sweep(u, rhs, diagonal, out, parameters, grid)`` with the same
arguments, each one launch over the three face lattices.
``HelmholtzWorkspace`` keeps the reference workspace's contract
(``mac/helmholtz.py:31-121``): a fixed count of sweeps from the diagonal
initial guess, optionally replayed from a captured CUDA graph (bounded LRU of
four counts), owned results.

The Stokes functions keep the signatures of ``mac/_triton_stokes.py``
(``start_partial``, ``residual_partial``, ``pressure_input_partial``,
``pressure_norm_partial``): one partial row per 256 cells in the caller's
buffer, reduced by the caller (``mac/stokes_workspace.py``).

CUDA only: CPU tensors are rejected.
"""
from collections import OrderedDict
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code, pointers, int64s, doubles


def _check_faces(tensors, what):
    for t in tensors:
        if not torch.is_tensor(t) or not t.is_cuda:
            raise ValueError(f'{what}: the B200 kernels need CUDA tensors; there is no CPU fallback')
        if not t.is_contiguous():
            raise ValueError(f'{what}: contiguous face arrays required')
    _lib.load()


class HelmholtzKernels:
    """Kernel object for ``HelmholtzWorkspace`` (``mac/_triton_helmholtz.py:62-77``)."""
    name = 'b200'

    def initialize(self, b, p, diagonal, rhs, u, parameters, grid):
        _check_faces((*b, *diagonal, *rhs, *u, parameters) + (() if p is None else (p,)), 'Helmholtz initialize')
        call('afsi_b200_helmholtz_initialize', pointers(b), ptr(p), pointers(diagonal), pointers(rhs), pointers(u),
             ptr(parameters), int64s(grid.shape), doubles(grid.spacing), dtype_code(b[0].dtype),
             stream(b[0].device))

    def sweep(self, u, rhs, diagonal, out, parameters, grid):
        _check_faces((*u, *rhs, *diagonal, *out, parameters), 'Helmholtz sweep')
        call('afsi_b200_helmholtz_sweep', pointers(u), pointers(rhs), pointers(diagonal), pointers(out),
             ptr(parameters), int64s(grid.shape), doubles([h * h for h in grid.spacing]), dtype_code(u[0].dtype),
             stream(u[0].device))


class HelmholtzWorkspace:
    """``mac/helmholtz.py:31-121`` on the B200 kernels: backend 'graph'
    (captured sweep chains, the reference default) or 'b200' (launched)."""

    def __init__(self, grid, diagonal, *, backend='graph', kernels=None):
        backend = {'triton': 'b200'}.get(backend, backend)
        if backend not in ('b200', 'graph'):
            raise ValueError('invalid Helmholtz workspace backend')
        _check_faces(diagonal, 'Helmholtz workspace')
        self.grid, self.diagonal, self.backend = grid, diagonal, backend
        self.rhs, self.first, self.second = [tuple(torch.empty_like(d) for d in diagonal) for _ in range(3)]
        self.parameters = diagonal[0].new_zeros(2)
        self._parameter_values = None
        self.kernels = kernels or HelmholtzKernels()
        self.graphs = OrderedDict()
        self._stream = None
        self.solves = self.sweeps = self.graph_builds = 0

    def _block(self, count):
        u, out = self.first, self.second
        for _ in range(count):
            self.kernels.sweep(u, self.rhs, self.diagonal, out, self.parameters, self.grid)
            u, out = out, u
        return u

    def _capture(self, count):
        if len(self.graphs) >= 4:
            self.graphs.popitem(last=False)
        dev = self.parameters.device
        with torch.cuda.device(dev):
            s = torch.cuda.Stream(device=dev)
            s.wait_stream(torch.cuda.current_stream(dev))
            g = torch.cuda.CUDAGraph()
            before = _lib.launch_count()
            with torch.cuda.graph(g, stream=s):
                self._block(count)
            self.graph_launches = _lib.launch_count() - before
            _lib.forget_launches(self.graph_launches)
            torch.cuda.current_stream(dev).wait_stream(s)
        self.graphs[count] = g
        self.graph_builds += 1

    @torch.no_grad()
    def solve(self, b, *, alpha, count, pressure=None, pressure_scale=0., owned=True):
        self.grid.check_velocity(b)
        if type(count) is not int or count < 1:
            raise ValueError('positive fixed Helmholtz iteration count required')
        if any(v.device != self.parameters.device or v.dtype != self.parameters.dtype for v in b):
            raise ValueError('Helmholtz workspace dtype/device mismatch')
        if pressure is not None and (pressure.shape != self.grid.shape or pressure.device != self.parameters.device
                                     or pressure.dtype != self.parameters.dtype):
            raise ValueError('Helmholtz pressure shape/device/dtype mismatch')
        s = torch.cuda.current_stream(self.parameters.device).cuda_stream
        if self._stream is not None and self._stream != s:
            raise ValueError('Helmholtz workspace requires its original CUDA stream')
        self._stream = s
        with torch.cuda.device(self.parameters.device):
            parameters = float(alpha), float(pressure_scale)
            if parameters != self._parameter_values:
                self.parameters[0].fill_(alpha)
                self.parameters[1].fill_(pressure_scale)
                self._parameter_values = parameters
            b = tuple(v.contiguous() for v in b)
            pressure = None if pressure is None else pressure.contiguous()
            if self.backend == 'graph' and count not in self.graphs:
                self._capture(count)
            self.kernels.initialize(b, pressure, self.diagonal, self.rhs, self.first, self.parameters, self.grid)
            if self.backend == 'graph':
                self.graphs.move_to_end(count)
                self.graphs[count].replay()
                _lib.count_replay(self.graph_launches)
                result = self.second if count % 2 else self.first
            else:
                result = self._block(count)
            self.solves += 1
            self.sweeps += count
            return tuple(v.clone() for v in result) if owned else result

    def summary(self):
        return dict(backend=self.backend, solves=self.solves, sweeps=self.sweeps, graph_builds=self.graph_builds,
                    cached_graphs=len(self.graphs),
                    buffer_bytes=sum(v.numel() * v.element_size() for group in (self.rhs, self.first, self.second)
                                     for v in group))


# ------------------------------------------------------------------ Stokes

def _blocks(shape, partial, width):
    n = _lib.load().afsi_b200_stokes_partial_blocks(int64s(shape))
    if n < 0:
        raise ValueError('invalid MAC grid shape')
    if tuple(partial.shape) != (n, width) and not (width == 1 and partial.numel() == n):
        raise ValueError(f'partial buffer must be ({n}, {width})')
    return n


def start_partial(b, p, partial, shape):
    """``mac/_triton_stokes.py:16-27,90-93``."""
    _check_faces((*b, p, partial), 'Stokes start')
    _blocks(shape, partial, 3)
    call('afsi_b200_stokes_start_partial', pointers(b), ptr(p), ptr(partial), int64s(shape), dtype_code(p.dtype),
         stream(p.device))


def residual_partial(u, p, b, residual, partial, shape, coefficients):
    """``mac/_triton_stokes.py:58-84,96-100``."""
    _check_faces((*u, p, *b, residual, partial, coefficients), 'Stokes residual')
    _blocks(shape, partial, 2)
    call('afsi_b200_stokes_residual_partial', pointers(u), ptr(p), pointers(b), ptr(residual), ptr(partial),
         ptr(coefficients), int64s(shape), dtype_code(p.dtype), stream(p.device))


def pressure_input_partial(rhs, p, partial):
    """``mac/_triton_stokes.py:103-114,135-138``."""
    _check_faces((rhs, p, partial), 'pressure input')
    n = p.numel()
    if tuple(partial.shape) != ((n + 255) // 256, 5):
        raise ValueError(f'partial buffer must be ({(n + 255) // 256}, 5)')
    call('afsi_b200_pressure_input_partial', ptr(rhs), ptr(p), n, ptr(partial), dtype_code(p.dtype),
         stream(p.device))


def pressure_norm_partial(rhs, p, partial, spacing_squared):
    """``mac/_triton_stokes.py:117-132,141-145``."""
    _check_faces((rhs, p, partial, spacing_squared), 'pressure norm')
    _blocks(p.shape, partial, 2)
    call('afsi_b200_pressure_norm_partial', ptr(rhs), ptr(p), ptr(partial), ptr(spacing_squared),
         int64s(p.shape), dtype_code(p.dtype), stream(p.device))
