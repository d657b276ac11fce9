"""MG-preconditioned FGMRES for the CN saddle point on the B200 kernels.

The reference solves  H u + (dt/rho) G p = b,  D u = 0  (H = I - alpha L,
alpha = dt mu / (2 rho)) with right-preconditioned restarted GMRES whose
preconditioner is a pressure-free projection: a fixed-count Jacobi Helmholtz
solve of the velocity part, then a multigrid pressure solve to a loose
tolerance (``mac/stokes_fgmres.py:15-96``, Krylov loop ``nonlinear.py:139-240``).
This module keeps that method, its tolerances and its acceptance test:

* ``CNStokes`` holds what the solve reads from the reference's CN flow
  (``mac/cnab.py:71-100``): grid, dt, rho, mu, alpha, the Helmholtz diagonal
  and sweep count, the pressure multigrid and the Stokes options.
* ``solve(flow, b, initial=None)`` follows ``stokes_fgmres.solve``: packed
  vectors [u0 | u1 | u2 | q], the operator action and the preconditioner as
  CUDA kernels of this library (``afsi_b200_stokes_action``,
  ``afsi_b200_stokes_precondition_rhs/_result``, the Helmholtz sweeps and the
  multigrid solve), the Krylov vectors and their dot products on the device.
* ``gmres(action, rhs, precondition=..., options=...)`` restates the reference's
  GMRES (two classical Gram-Schmidt passes, Givens estimate with periodic true
  residual checks, restart from the measured residual when an estimate is
  rejected).  The small Hessenberg system lives on the host; one host read of
  its new column per iteration (the reference reads it too).

Precision form (``precision='fp32-preconditioner'``): the preconditioner's
Helmholtz sweeps and V-cycles run in FP32 (FP64 coarsest solve), while the
outer FGMRES residuals, the operator action and the update stay FP64; the
flexible Krylov method absorbs the inexact preconditioner, and acceptance
is the reference's FP64 true-residual test.
"""
from dataclasses import dataclass
from math import ceil, isfinite, log
import numpy as np
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code, int64s, doubles
from .helmholtz import HelmholtzSolver, residual_partial
from .multigrid import GeometricMultigrid, MGOptions


@dataclass(frozen=True)
class GMRESOptions:
    """``nonlinear.py:14-31``."""
    rtol: float = 1e-3
    atol: float = 1e-12
    restart: int = 50
    max_iterations: int = 1000
    check_every: int = 5
    check_policy: str = 'periodic'
    true_check_interval: int = 25

    def __post_init__(self):
        if not all(isfinite(t) and t >= 0 for t in (self.rtol, self.atol)) or self.rtol + self.atol == 0:
            raise ValueError('invalid linear tolerances')
        for n in (self.restart, self.max_iterations, self.check_every, self.true_check_interval):
            if not isinstance(n, int) or isinstance(n, bool) or n < 1:
                raise ValueError('positive integer GMRES controls required')
        if self.check_policy not in ('periodic', 'estimated'):
            raise ValueError('GMRES check_policy must be periodic or estimated')


class KrylovSpace:
    """Arnoldi storage reused across solves: the basis V and the
    preconditioned directions Z as rows of two device matrices, so each vector
    is contiguous and the projections are matrix-vector products."""

    def __init__(self):
        self.key = None
        self.allocations = 0

    def vectors(self, rhs, width):
        key = (rhs.numel(), width, rhs.dtype, rhs.device)
        if key != self.key:
            self.V = rhs.new_empty((width + 1, rhs.numel()))
            self.Z = rhs.new_empty((width, rhs.numel()))
            self.key = key
            self.allocations += 1
        return self.V, self.Z


@torch.no_grad()
def gmres(action, rhs, *, precondition=None, options=None, workspace=None):
    """Restarted right-preconditioned GMRES from zero (``nonlinear.py:139-240``);
    residuals use the original operator; returns (x, info)."""
    opt = GMRESOptions() if options is None else options
    if rhs.dtype not in (torch.float32, torch.float64) or not rhs.numel():
        raise ValueError('nonempty floating rhs required')
    b = rhs.reshape(-1)
    eps, tiny = torch.finfo(b.dtype).eps, torch.finfo(b.dtype).tiny
    norm = lambda x: torch.linalg.vector_norm(x).item()
    tol = max(opt.atol, opt.rtol * norm(b))
    stats = dict(actions=0, true=0, estimated=0, restarts=0)

    def apply(v):
        stats['actions'] += 1
        out = action(v.reshape(rhs.shape)).reshape(-1)
        if out.shape != b.shape or out.dtype != b.dtype or out.device != b.device:
            raise ValueError('GMRES operator action shape/dtype/device mismatch')
        return out

    def solve_pre(v):
        out = v if precondition is None else precondition(v.reshape(rhs.shape)).reshape(-1)
        if out.shape != b.shape or out.dtype != b.dtype or out.device != b.device:
            raise ValueError('GMRES preconditioner action shape/dtype/device mismatch')
        return out

    x = torch.zeros_like(b)
    residual = b - apply(x)
    res_norm = norm(residual)
    count = 0

    def info():
        return dict(iterations=count, residual_norm=res_norm, tolerance=tol, operator_actions=stats['actions'],
                    true_residual_checks=stats['true'], estimated_residual_checks=stats['estimated'],
                    residual_restarts=stats['restarts'])

    while res_norm > tol and count < opt.max_iterations:
        beta = res_norm
        width = min(opt.restart, opt.max_iterations - count, b.numel())
        if workspace is None:
            V, Z = b.new_empty((width + 1, b.numel())), b.new_empty((width, b.numel()))
        else:
            V, Z = workspace.vectors(b, width)
        H = np.zeros((width + 1, width))
        Hd = b.new_zeros((width + 1, width))
        estimated = opt.check_policy == 'estimated'
        rotated = np.zeros((width + 1, width))
        cos, sin = np.zeros(width), np.zeros(width)
        g = np.zeros(width + 1)
        g[0] = beta
        V[0] = residual / beta
        base = x.clone()
        for j in range(width):
            Z[j] = solve_pre(V[j])
            w = apply(Z[j])
            original = torch.linalg.vector_norm(w)
            for _ in range(2):  # classical Gram-Schmidt, twice
                coefficients = torch.mv(V[:j + 1], w)
                Hd[:j + 1, j] += coefficients
                w = w - torch.mv(V[:j + 1].t(), coefficients)
            Hd[j + 1, j] = torch.linalg.vector_norm(w)
            column = torch.cat((Hd[:j + 2, j], original.reshape(1))).tolist()  # one host read
            H[:j + 2, j] = column[:j + 2]
            breakdown = H[j + 1, j] <= 100 * eps * max(column[-1], tiny)
            if not breakdown:
                V[j + 1] = w / Hd[j + 1, j]
            count += 1
            converged_estimate = False
            if estimated:
                col = H[:j + 2, j].copy()
                for k in range(j):
                    a, c = col[k], col[k + 1]
                    col[k] = cos[k] * a + sin[k] * c
                    col[k + 1] = -sin[k] * a + cos[k] * c
                radius = np.hypot(col[j], col[j + 1])
                den = max(radius, tiny)
                cos[j], sin[j] = col[j] / den, col[j + 1] / den
                col[j], col[j + 1] = radius, 0.
                rotated[:j + 2, j] = col
                previous = g[j]
                g[j + 1], g[j] = -sin[j] * previous, cos[j] * previous
                stats['estimated'] += 1
                converged_estimate = abs(g[j + 1]) <= tol
            scheduled = (j + 1) % opt.check_every == 0 if not estimated else count % opt.true_check_interval == 0
            if breakdown or scheduled or converged_estimate or j + 1 == width:
                Q, R = np.linalg.qr(H[:j + 2, :j + 1], mode='reduced')
                if (np.abs(np.diag(R)) <= eps * np.abs(R).max()).any():
                    raise RuntimeError('GMRES singular Hessenberg system')
                target = np.zeros(j + 2)
                target[0] = beta
                y = np.linalg.solve(R, Q.T @ target)
                x = base + torch.mv(Z[:j + 1].t(), torch.as_tensor(y, device=b.device, dtype=b.dtype))
                residual = b - apply(x)
                res_norm = norm(residual)
                stats['true'] += 1
                if res_norm <= tol:
                    return x.reshape(rhs.shape), info()
                if breakdown:
                    raise RuntimeError('GMRES breakdown before true-residual convergence')
                if converged_estimate:
                    stats['restarts'] += 1  # a rejected estimate restarts from the measured residual
                    break
    if res_norm > tol:
        raise RuntimeError(f'GMRES failed: true residual {res_norm:.6g} > {tol:.6g} after {count} iterations')
    return x.reshape(rhs.shape), info()


@dataclass(frozen=True)
class StokesResult:
    velocity: tuple
    pressure: torch.Tensor
    diagnostics: dict


class CNStokes:
    """The CN flow parameters and solvers the FGMRES solve uses
    (``mac/cnab.py:71-100``): H = I - alpha L with alpha = dt mu / (2 rho), its
    Jacobi diagonal and the fixed sweep count that reaches helmholtz_rtol, the
    pressure multigrid (``GeometricMultigrid``) and the Stokes options
    (restart 20, at most 40 iterations, preconditioner tolerance 0.01)."""

    def __init__(self, grid, *, dt, rho=1., mu=1., device='cuda', options=None, helmholtz_rtol=1e-13,
                 max_helmholtz_iterations=512, stokes_restart=20, max_stokes_iterations=40,
                 stokes_preconditioner_rtol=.01, precision='fp64'):
        if any(not isfinite(v) or v <= 0 for v in (dt, rho, mu)):
            raise ValueError('positive dt/rho/mu required')
        if precision not in ('fp64', 'fp32-preconditioner'):
            raise ValueError("precision must be 'fp64' or 'fp32-preconditioner'")
        if not 0 < stokes_preconditioner_rtol < 1:
            raise ValueError('stokes_preconditioner_rtol must lie in (0, 1)')
        device = torch.device(device)
        if device.type != 'cuda':
            raise ValueError('the B200 Stokes solve requires a CUDA device; there is no CPU fallback')
        self.grid, self.dt, self.rho, self.mu = grid, float(dt), float(rho), float(mu)
        self.alpha = self.dt * self.mu / (2 * self.rho)
        self.options = MGOptions() if options is None else options
        self.restart, self.max_iterations = int(stokes_restart), int(max_stokes_iterations)
        self.preconditioner_rtol = float(stokes_preconditioner_rtol)
        self.precision = precision
        s = 2 * self.alpha * sum(1 / h ** 2 for h in grid.spacing)
        q = s / (1 + s)
        self.helmholtz_iterations = max(1, ceil(log(helmholtz_rtol / (1 + s)) / log(q))) if q else 1
        if self.helmholtz_iterations > max_helmholtz_iterations:
            raise ValueError('CN Helmholtz iteration budget too small for this dt/viscosity/grid')
        self.diagonal = self._diagonal(device)
        pre_dtype = torch.float64 if precision == 'fp64' else torch.float32
        self.pressure_solver = GeometricMultigrid(grid, device=device, dtype=pre_dtype, options=self.options,
                                                  coarse_dtype=torch.float64)
        self.helmholtz = HelmholtzSolver(grid, tuple(d.to(pre_dtype) for d in self.diagonal), self.alpha,
                                         self.helmholtz_iterations)
        if precision == 'fp64':
            self.helmholtz64 = self.helmholtz
        else:
            self.helmholtz64 = HelmholtzSolver(grid, self.diagonal, self.alpha, self.helmholtz_iterations)
        self._shape = int64s(grid.shape)
        self._spacing = doubles(grid.spacing)
        lib = _lib.load()
        self.size = int(lib.afsi_b200_stokes_packed_size(self._shape))
        self.cells = int(np.prod(grid.shape))
        self.faces = self.size - self.cells
        self.face_sizes = [int(np.prod(grid.face_shape(c))) for c in range(3)]
        self.scratch = torch.zeros(int(lib.afsi_b200_stokes_precondition_scratch_bytes(self._shape)), device=device,
                                   dtype=torch.uint8)
        self.sums = torch.zeros(8, device=device, dtype=torch.float64)
        self.krylov = KrylovSpace()
        self.stokes_calls = 0

    def _diagonal(self, device):
        """``mac/cnab.py:82-92``."""
        out = []
        base = 1 + 2 * self.alpha * sum(1 / h ** 2 for h in self.grid.spacing)
        for c in range(3):
            d = torch.full(self.grid.face_shape(c), base, device=device, dtype=torch.float64)
            for axis, h in enumerate(self.grid.spacing):
                if axis != c:
                    d.narrow(axis, 0, 1).add_(self.alpha / h ** 2)
                    d.narrow(axis, d.shape[axis] - 1, 1).add_(self.alpha / h ** 2)
            d.narrow(c, 0, 1).fill_(1.)
            d.narrow(c, d.shape[c] - 1, 1).fill_(1.)
            out.append(d)
        return tuple(out)

    # -- packed vectors
    def unpack(self, v):
        parts = v.reshape(-1).split((*self.face_sizes, self.cells))
        return tuple(z.view(self.grid.face_shape(c)) for c, z in enumerate(parts[:3])), parts[3].view(self.grid.shape)

    def pack(self, u, q, out=None):
        out = torch.empty(self.size, device=q.device, dtype=q.dtype) if out is None else out
        torch.cat([t.reshape(-1) for t in u] + [q.reshape(-1)], out=out)
        return out

    def stokes(self, b, initial=None):
        return solve(self, b, initial)

    def metrics(self, u, p, b):
        """[||u - alpha L u + (dt/rho) G p - b||, ||D u||] (``mac/cnab.py:207-214``)."""
        scale = self.dt / self.rho
        coef = torch.tensor([self.alpha, scale, 1 / scale, *(1 / h for h in self.grid.spacing),
                             *(1 / (h * h) for h in self.grid.spacing)], device=p.device, dtype=p.dtype)
        blocks = _lib.load().afsi_b200_stokes_partial_blocks(self._shape)
        partial = torch.empty((blocks, 2), device=p.device, dtype=torch.float64)
        residual = torch.empty_like(p)
        residual_partial(u, p, b, residual, partial, self.grid.shape, coef)
        return partial.sum(0).sqrt()


def _precondition(flow, v, h):
    """pack(t - G phi, (phi + alpha rhs)/h - mean) for t = Helmholtz(r),
    rhs = (-s)/h - D t - mean, phi = multigrid solve of rhs to the
    preconditioner tolerance (``mac/stokes_fgmres.py:46-63``)."""
    work = v if flow.precision == 'fp64' else v.float()
    r, s = flow.unpack(work)
    tentative = flow.helmholtz.solve(r, out=None)
    st = stream(v.device)
    code = dtype_code(work.dtype)
    rhs = torch.empty(flow.grid.shape, device=v.device, dtype=work.dtype)
    tp = ctypes_ptrs(tentative)
    call('afsi_b200_stokes_precondition_rhs', tp, ptr(s), ptr(rhs), ptr(flow.sums), ptr(flow.scratch), flow._shape,
         flow._spacing, h, code, st)
    call('afsi_b200_subtract_mean', ptr(rhs), rhs.numel(), ptr(flow.sums), code, st)
    phi, info = flow.pressure_solver.solve(rhs, rtol=flow.preconditioner_rtol)
    out = torch.empty(flow.size, device=v.device, dtype=work.dtype)
    call('afsi_b200_stokes_precondition_result', tp, ptr(phi), ptr(rhs), ptr(out), ptr(flow.sums[1:]),
         ptr(flow.scratch), flow._shape, flow._spacing, flow.alpha, h, code, st)
    q = out[flow.faces:]
    call('afsi_b200_subtract_mean', ptr(q), q.numel(), ptr(flow.sums[1:]), code, st)
    return (out if flow.precision == 'fp64' else out.double()), info['cycles']


def ctypes_ptrs(faces):
    import ctypes
    return (ctypes.c_void_p * 3)(*[t.data_ptr() for t in faces])


@torch.no_grad()
def solve(flow, b, initial=None):
    """``mac/stokes_fgmres.py:15-96`` on the B200: returns a ``StokesResult``
    (velocity, pressure, diagnostics with the reference's keys)."""
    flow.stokes_calls += 1
    grid = flow.grid
    grid.check_velocity(b)
    dev = b[0].device
    if b[0].dtype != torch.float64:
        raise ValueError('the CN Stokes solve is FP64 (the precision form changes the preconditioner only)')
    b = tuple(v.clone() for v in b)
    for c, v in enumerate(b):  # zero_normal
        v.narrow(c, 0, 1).zero_()
        v.narrow(c, v.shape[c] - 1, 1).zero_()
    if initial is None:
        p = torch.zeros(grid.shape, device=dev, dtype=torch.float64)
    else:
        if tuple(initial.shape) != tuple(grid.shape) or initial.device != dev or initial.dtype != torch.float64 \
                or not torch.isfinite(initial).all():
            raise ValueError('invalid initial CN Stokes pressure')
        p = initial.clone()
    p -= p.mean()
    h = min(grid.spacing)
    scale = flow.dt / flow.rho
    alpha = flow.alpha
    st = stream(dev)
    shape, spacing = flow._shape, flow._spacing

    def action(v):
        out = torch.empty_like(v)
        call('afsi_b200_stokes_action', ptr(v), ptr(out), shape, spacing, alpha, h, _lib.F64, st)
        return out

    counters = dict(poisson_solves=0, cycles=0)

    def precondition(v):
        out, cycles = _precondition(flow, v.contiguous(), h)
        counters['poisson_solves'] += 1
        counters['cycles'] += cycles
        return out

    norm_b = torch.sqrt(sum(v.square().sum() for v in b)).item()
    if not isfinite(norm_b):
        raise ValueError('nonfinite CN Stokes RHS')
    opt = flow.pressure_solver.options
    momentum_tol = max(opt.atol, opt.rtol * norm_b)
    z = flow.helmholtz64.solve(b)
    zero_q = torch.zeros(grid.shape, device=dev, dtype=torch.float64)
    negdiv = torch.empty(grid.shape, device=dev, dtype=torch.float64)
    # (-0)/h - D z = -D z exactly
    call('afsi_b200_stokes_precondition_rhs', ctypes_ptrs(z), ptr(zero_q), ptr(negdiv), ptr(flow.sums),
         ptr(flow.scratch), shape, spacing, h, _lib.F64, st)
    div_rhs = negdiv / scale
    div_tol = scale * max(opt.atol, opt.rtol * torch.linalg.vector_norm(div_rhs).item())
    floor = 100 * torch.finfo(torch.float64).eps * max(norm_b, torch.finfo(torch.float64).tiny) * \
        sum(1 / d for d in grid.spacing)
    div_tol = max(div_tol, floor)
    initial_u = flow.helmholtz64.solve(b, p, scale)
    guess = flow.pack(initial_u, scale / h * p)
    target = flow.pack(b, zero_q)
    rhs = target - action(guess)
    tolerance = .5 * min(momentum_tol, h * div_tol)
    controls = GMRESOptions(rtol=0., atol=tolerance, restart=flow.restart, max_iterations=flow.max_iterations,
                            check_policy='estimated', true_check_interval=5)
    correction, info = gmres(action, rhs, precondition=precondition, options=controls, workspace=flow.krylov)
    u, q = flow.unpack(guess + correction)
    p = h / scale * (q - q.mean())
    u = tuple(t.contiguous() for t in u)
    momentum, divn = flow.metrics(u, p, b).tolist()
    if momentum > momentum_tol or divn > div_tol:
        raise RuntimeError(f'CN FGMRES true residual rejected: momentum {momentum}/{momentum_tol}, '
                           f'divergence {divn}/{div_tol}')
    return StokesResult(u, p, dict(
        pressure=dict(cycles=counters['cycles'], backend=flow.pressure_solver.backend,
                      poisson_solves=counters['poisson_solves'], schur_iterations=info['iterations'],
                      residual_norm=divn / scale, tolerance=div_tol / scale,
                      meaning='CN half-time pressure; coupled saddle-point solve'),
        stokes=dict(momentum_residual=momentum, momentum_tolerance=momentum_tol, divergence_norm=divn,
                    divergence_tolerance=div_tol, solver='fgmres',
                    preconditioner='pressure-free projection with geometric MG', iterations=info['iterations'],
                    operator_actions=info['operator_actions'], preconditioner_rtol=flow.preconditioner_rtol,
                    helmholtz_iterations=flow.helmholtz_iterations, precision=flow.precision)))
