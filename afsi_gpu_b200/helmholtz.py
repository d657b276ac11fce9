"""CN Helmholtz Jacobi sweeps and Stokes residual reductions on the B200.

``HelmholtzKernels`` is the kernel object of ``mac/helmholtz.py``'s
``HelmholtzWorkspace`` (the reference builds ``_triton_helmholtz.HelmholtzKernels``,
``mac/helmholtz.py:44-47``): ``initialize(b, p, diagonal, rhs, u, parameters,
grid)`` and ``sweep(u, rhs, diagonal, out, parameters, grid)`` with the same
arguments, each one launch over the three face lattices.
``HelmholtzSolver`` runs a fixed-count solve (initialize plus sweeps) as one
captured graph over staged inputs; the reference's own ``HelmholtzWorkspace``
runs on ``HelmholtzKernels`` after ``dropin.install()``.

The Stokes functions keep the signatures of ``mac/_triton_stokes.py``
(``start_partial``, ``residual_partial``, ``pressure_input_partial``,
``pressure_norm_partial``): one partial row per 256 cells in the caller's
buffer, reduced by the caller (``mac/stokes_workspace.py``).

CUDA only: CPU tensors are rejected.
"""
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


class HelmholtzSolver:
    """Fixed-count CN Helmholtz solve on the B200 kernels.

    Solves (I - alpha L) u = b - pressure_scale * G p approximately, the way
    the reference's CN flow does (``mac/cnab.py:176-192``): the initial guess
    rhs/diagonal, then `count` Jacobi sweeps, wall-normal faces held at zero.

    The design is this package's own.  `alpha` and `count` are fixed for the
    solver's life (a CN flow changes them only with its time step).  The
    right-hand side and the pressure are staged into the solver's own input
    buffers (``inputs``), so with ``graph=True`` the whole chain (the
    initialize launch and every sweep) is one CUDA graph per pressure mode,
    captured on first use and replayed afterwards; ``graph=False`` launches
    the same kernels.  A caller that fills ``inputs`` itself passes
    ``staged=True`` and skips the copies.  Results are returned as fresh
    tensors unless ``out`` is given.  One solver serves one stream at a time.
    """

    def __init__(self, grid, diagonal, alpha, count, *, graph=True, kernels=None):
        if type(count) is not int or count < 1:
            raise ValueError('the Helmholtz sweep count must be a positive integer')
        diagonal = tuple(diagonal)
        _check_faces(diagonal, 'Helmholtz solver')
        grid.check_velocity(diagonal)
        ref = diagonal[0]
        self.grid, self.diagonal, self.count, self.alpha = grid, diagonal, count, float(alpha)
        self.kernels = kernels or HelmholtzKernels()
        self.use_graph = bool(graph)
        faces = lambda: tuple(torch.zeros_like(d) for d in diagonal)
        self.inputs = faces()
        self.pressure = torch.zeros(grid.shape, device=ref.device, dtype=ref.dtype)
        self._rhs, self._ping, self._pong = faces(), faces(), faces()
        self._param = torch.tensor([self.alpha, 0.], device=ref.device, dtype=ref.dtype)
        self._scale = 0.
        self._graphs = {}
        self._launches = {}
        self.calls = 0

    @property
    def result(self):
        """The buffer the last sweep writes (ping after an even count)."""
        return self._ping if self.count % 2 == 0 else self._pong

    def _chain(self, with_pressure):
        self.kernels.initialize(self.inputs, self.pressure if with_pressure else None, self.diagonal, self._rhs,
                                self._ping, self._param, self.grid)
        src, dst = self._ping, self._pong
        for _ in range(self.count):
            self.kernels.sweep(src, self._rhs, self.diagonal, dst, self._param, self.grid)
            src, dst = dst, src

    def _graph(self, with_pressure):
        if with_pressure not in self._graphs:
            dev = self._param.device
            with torch.cuda.device(dev):
                side = torch.cuda.Stream(device=dev)
                side.wait_stream(torch.cuda.current_stream(dev))
                g = torch.cuda.CUDAGraph()
                before = _lib.launch_count()
                with torch.cuda.graph(g, stream=side):
                    self._chain(with_pressure)
                self._launches[with_pressure] = _lib.launch_count() - before
                _lib.forget_launches(self._launches[with_pressure])
                torch.cuda.current_stream(dev).wait_stream(side)
            self._graphs[with_pressure] = g
        return self._graphs[with_pressure]

    @torch.no_grad()
    def solve(self, b=None, pressure=None, pressure_scale=0., *, staged=False, out=None):
        """u for right-hand side `b` (face arrays) and, optionally, the pressure
        term; with staged=True, `b` and `pressure` were written into
        ``inputs`` / ``pressure`` already (pass pressure=True to use it)."""
        with_pressure = pressure is not None and pressure is not False
        if not staged:
            self.grid.check_velocity(b)
            ref = self.inputs[0]
            if b[0].dtype != ref.dtype or b[0].device != ref.device:
                raise ValueError('Helmholtz right-hand side dtype/device differs from the solver\'s')
            for dst, src in zip(self.inputs, b):
                dst.copy_(src)
            if with_pressure:
                if tuple(pressure.shape) != tuple(self.grid.shape) or pressure.dtype != ref.dtype:
                    raise ValueError('Helmholtz pressure shape/dtype mismatch')
                self.pressure.copy_(pressure)
        if with_pressure and float(pressure_scale) != self._scale:
            self._scale = float(pressure_scale)
            self._param[1].fill_(self._scale)
        if self.use_graph:
            self._graph(with_pressure).replay()
            _lib.count_replay(self._launches[with_pressure])
        else:
            self._chain(with_pressure)
        self.calls += 1
        res = self.result
        if out is None:
            return tuple(v.clone() for v in res)
        for o, v in zip(out, res):
            o.copy_(v)
        return out


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
