"""NumPy restatement of the CN Helmholtz sweeps and the Stokes residual
reductions (oracle; test infrastructure only).

* ``helmholtz_initialize`` / ``helmholtz_sweep``: ``TorchHelmholtzKernels``,
  ``mac/helmholtz.py:14-28``, with ``gradient``, ``zero_normal`` and
  ``velocity_laplacian`` of ``mac/grid.py:62-105``.
* ``stokes_start`` / ``stokes_measure``: the buffered CPU branches of
  ``StokesWorkspace.start/measure``, ``mac/stokes_workspace.py:79-105``.
* ``pressure_metrics``: the sums ``PressureStartMetrics`` reduces,
  ``mac/stokes_workspace.py:20-55`` with ``mac/_triton_stokes.py:103-132``.
"""
import numpy as np


def _slab(axis, start=None, stop=None):
    key = [slice(None)] * 3
    key[axis] = slice(start, stop)
    return tuple(key)


def gradient(p, spacing):
    out = []
    for c, h in enumerate(spacing):
        shape = list(p.shape)
        shape[c] += 1
        g = np.zeros(shape, dtype=p.dtype)
        g[_slab(c, 1, -1)] = np.diff(p, axis=c) / p.dtype.type(h)
        out.append(g)
    return out


def zero_normal(velocity):
    out = [u.copy() for u in velocity]
    for c, u in enumerate(out):
        u[_slab(c, 0, 1)] = 0
        u[_slab(c, -1, None)] = 0
    return out


def velocity_laplacian(u, component, spacing):
    out = np.zeros_like(u)
    for axis, h in enumerate(spacing):
        left = np.concatenate((-u[_slab(axis, 0, 1)], u[_slab(axis, None, -1)]), axis)
        right = np.concatenate((u[_slab(axis, 1, None)], -u[_slab(axis, -1, None)]), axis)
        out = out + (left - 2 * u + right) / u.dtype.type(h * h)
    out[_slab(component, 0, 1)] = 0
    out[_slab(component, -1, None)] = 0
    return out


def helmholtz_initialize(b, p, diagonal, pressure_scale, spacing):
    """(rhs, u): rhs = zero_normal(b - s G p), u = rhs / diag."""
    if p is not None:
        s = b[0].dtype.type(pressure_scale)
        b = [r - s * g for r, g in zip(b, gradient(p, spacing))]
    rhs = zero_normal(b)
    return rhs, [r / d for r, d in zip(rhs, diagonal)]


def helmholtz_sweep(u, rhs, diagonal, alpha, spacing):
    a = u[0].dtype.type(alpha)
    return zero_normal([v + (r - v + a * velocity_laplacian(v, c, spacing)) / d
                        for c, (v, r, d) in enumerate(zip(u, rhs, diagonal))])


def divergence(velocity, spacing):
    return sum(np.diff(u, axis=c) / u.dtype.type(spacing[c]) for c, u in enumerate(velocity))


def stokes_start(b, p):
    """[||b||, mean p, all p finite]."""
    return np.array([np.sqrt(sum((v.astype(np.float64) ** 2).sum() for v in b)), p.mean(dtype=np.float64),
                     float(np.isfinite(p).all())])


def stokes_measure(u, p, b, alpha, dt_over_rho, spacing):
    """([||momentum residual||, ||D u||], residual = -(rho/dt) D u)."""
    gp = gradient(p, spacing)
    a, s = u[0].dtype.type(alpha), u[0].dtype.type(dt_over_rho)
    momentum = [v - a * velocity_laplacian(v, c, spacing) + s * g - r
                for c, (v, g, r) in enumerate(zip(u, gp, b))]
    div = divergence(u, spacing)
    norms = np.array([np.sqrt(sum((m.astype(np.float64) ** 2).sum() for m in momentum)),
                      np.sqrt((div.astype(np.float64) ** 2).sum())])
    return norms, -u[0].dtype.type(1 / dt_over_rho) * div


def neg_laplacian(p, spacing):
    """``mac/grid.py:86-93``."""
    out = np.zeros_like(p)
    for c, h in enumerate(spacing):
        d = np.diff(p, axis=c) / p.dtype.type(h * h)
        out[_slab(c, None, -1)] -= d
        out[_slab(c, 1, None)] += d
    return out


def pressure_metrics(rhs, p, spacing):
    """[sum rhs, sum |rhs|, sum p, rhs finite, p finite, ||rhs||, ||rhs - A p||]."""
    r64 = rhs.astype(np.float64)
    res = (rhs - neg_laplacian(p, spacing)).astype(np.float64)
    return np.array([r64.sum(), np.abs(r64).sum(), p.astype(np.float64).sum(), float(np.isfinite(rhs).all()),
                     float(np.isfinite(p).all()), np.sqrt((r64 ** 2).sum()), np.sqrt((res ** 2).sum())])


# ----------------------------------------------------------- FGMRES Stokes
# mac/stokes_fgmres.py:15-96 with the Krylov loop of nonlinear.py:139-240 and
# the CN flow pieces of mac/cnab.py:71-100,176-192,207-214.

def cn_diagonal(shape, spacing, alpha):
    """Jacobi diagonal of H = I - alpha L per face lattice (``mac/cnab.py:82-92``)."""
    base = 1 + 2 * alpha * sum(1 / h ** 2 for h in spacing)
    out = []
    for c in range(3):
        fs = list(shape)
        fs[c] += 1
        d = np.full(fs, base)
        for axis, h in enumerate(spacing):
            if axis != c:
                d[_slab(axis, 0, 1)] += alpha / h ** 2
                d[_slab(axis, -1, None)] += alpha / h ** 2
        d[_slab(c, 0, 1)] = 1.
        d[_slab(c, -1, None)] = 1.
        out.append(d)
    return out


def helmholtz_count(alpha, spacing, rtol=1e-13):
    """Fixed Jacobi sweep count (``mac/cnab.py:95-97``)."""
    from math import ceil, log
    s = 2 * alpha * sum(1 / h ** 2 for h in spacing)
    q = s / (1 + s)
    return max(1, ceil(log(rtol / (1 + s)) / log(q))) if q else 1


def helmholtz_solve(b, diagonal, alpha, count, spacing, p=None, scale=0.):
    """``MACCNABFlow._solve_helmholtz`` (``mac/cnab.py:181-192``)."""
    rhs, u = helmholtz_initialize(b, p, diagonal, scale, spacing)
    for _ in range(count):
        u = helmholtz_sweep(u, rhs, diagonal, alpha, spacing)
    return u


class StokesProblem:
    """The packed saddle-point operator and its preconditioner."""

    def __init__(self, shape, spacing, dt, rho, mu, hierarchy, *, preconditioner_rtol=.01):
        from . import mg
        self.shape, self.spacing = tuple(shape), tuple(spacing)
        self.dt, self.rho, self.mu = dt, rho, mu
        self.alpha = dt * mu / (2 * rho)
        self.h = min(spacing)
        self.scale = dt / rho
        self.diagonal = cn_diagonal(shape, spacing, self.alpha)
        self.count = helmholtz_count(self.alpha, spacing)
        self.hierarchy = hierarchy
        self.mg = mg
        self.pre_rtol = preconditioner_rtol
        self.face_shapes = [tuple(n + (a == c) for a, n in enumerate(shape)) for c in range(3)]
        self.sizes = [int(np.prod(s)) for s in self.face_shapes] + [int(np.prod(shape))]
        self.poisson_solves = self.cycles = 0

    def pack(self, u, q):
        return np.concatenate([x.reshape(-1) for x in u] + [q.reshape(-1)])

    def unpack(self, v):
        parts = np.split(v, np.cumsum(self.sizes)[:-1])
        return [p.reshape(s) for p, s in zip(parts[:3], self.face_shapes)], parts[3].reshape(self.shape)

    def helmholtz(self, b, p=None):
        return helmholtz_solve(b, self.diagonal, self.alpha, self.count, self.spacing, p, self.scale)

    def action(self, v):
        """``stokes_fgmres.py:36-43``."""
        u, q = self.unpack(v)
        gp = gradient(q, self.spacing)
        hu = [a - self.alpha * velocity_laplacian(a, c, self.spacing) + self.h * g
              for c, (a, g) in enumerate(zip(u, gp))]
        return self.pack(zero_normal(hu), -self.h * divergence(u, self.spacing))

    def precondition(self, v):
        """``stokes_fgmres.py:46-63``."""
        r, s = self.unpack(v)
        tentative = self.helmholtz(r)
        rhs = -s / self.h - divergence(tentative, self.spacing)
        rhs = rhs - rhs.mean()
        phi, info = self.mg.solve(self.hierarchy, rhs, rtol=self.pre_rtol)
        self.poisson_solves += 1
        self.cycles += info['cycles']
        grad = gradient(phi, self.spacing)
        q = (phi + self.alpha * rhs) / self.h
        return self.pack([a - g for a, g in zip(tentative, grad)], q - q.mean())

    def metrics(self, u, p, b):
        """``mac/cnab.py:207-214``."""
        gp = gradient(p, self.spacing)
        momentum = [v - self.alpha * velocity_laplacian(v, c, self.spacing) + self.scale * g - r
                    for c, (v, g, r) in enumerate(zip(u, gp, b))]
        return (np.sqrt(sum((m ** 2).sum() for m in momentum)),
                np.linalg.norm(divergence(u, self.spacing).reshape(-1)))


def gmres(action, b, precondition, tol, restart, max_iterations, true_check_interval=5):
    """Restarted right-preconditioned GMRES from zero, 'estimated' check policy
    (``nonlinear.py:139-240``).  Returns (x, info)."""
    eps, tiny = np.finfo(np.float64).eps, np.finfo(np.float64).tiny
    actions = [0]

    def apply(v):
        actions[0] += 1
        return action(v)

    x = np.zeros_like(b)
    residual = b - apply(x)
    count = 0
    while np.linalg.norm(residual) > tol and count < max_iterations:
        beta = np.linalg.norm(residual)
        width = min(restart, max_iterations - count, b.size)
        V = np.zeros((b.size, width + 1))
        Z = np.zeros((b.size, width))
        H = np.zeros((width + 1, width))
        cos, sin, g = np.zeros(width), np.zeros(width), np.zeros(width + 1)
        g[0] = beta
        V[:, 0] = residual / beta
        base = x.copy()
        for j in range(width):
            Z[:, j] = precondition(V[:, j])
            w = apply(Z[:, j])
            original = np.linalg.norm(w)
            for _ in range(2):
                coefficients = V[:, :j + 1].T @ w
                H[:j + 1, j] += coefficients
                w = w - V[:, :j + 1] @ coefficients
            H[j + 1, j] = np.linalg.norm(w)
            breakdown = H[j + 1, j] <= 100 * eps * max(original, tiny)
            if not breakdown:
                V[:, j + 1] = w / H[j + 1, j]
            count += 1
            col = H[:j + 2, j].copy()
            for k in range(j):
                a, c = col[k], col[k + 1]
                col[k] = cos[k] * a + sin[k] * c
                col[k + 1] = -sin[k] * a + cos[k] * c
            radius = np.hypot(col[j], col[j + 1])
            den = max(radius, tiny)
            cos[j], sin[j] = col[j] / den, col[j + 1] / den
            previous = g[j]
            g[j + 1], g[j] = -sin[j] * previous, cos[j] * previous
            estimated = abs(g[j + 1]) <= tol
            if breakdown or count % true_check_interval == 0 or estimated or j + 1 == width:
                Q, R = np.linalg.qr(H[:j + 2, :j + 1])
                if (np.abs(np.diag(R)) <= eps * np.abs(R).max()).any():
                    raise RuntimeError('GMRES singular Hessenberg system')
                target = np.zeros(j + 2)
                target[0] = beta
                y = np.linalg.solve(R, Q.T @ target)
                x = base + Z[:, :j + 1] @ y
                residual = b - apply(x)
                if np.linalg.norm(residual) <= tol:
                    return x, dict(iterations=count, operator_actions=actions[0])
                if breakdown:
                    raise RuntimeError('GMRES breakdown before true-residual convergence')
                if estimated:
                    break
    if np.linalg.norm(residual) > tol:
        raise RuntimeError('GMRES failed')
    return x, dict(iterations=count, operator_actions=actions[0])


def fgmres_solve(problem, b, initial=None, *, rtol=1e-10, atol=1e-12, restart=20, max_iterations=40):
    """``stokes_fgmres.solve`` (``mac/stokes_fgmres.py:15-96``): returns
    (u, p, info) with the reference's counters and residual metrics."""
    P = problem
    b = zero_normal([np.asarray(v, dtype=np.float64) for v in b])
    p = np.zeros(P.shape) if initial is None else np.array(initial, dtype=np.float64)
    p = p - p.mean()
    h, scale = P.h, P.scale
    norm_b = np.sqrt(sum((v ** 2).sum() for v in b))
    momentum_tol = max(atol, rtol * norm_b)
    z = P.helmholtz(b)
    div_rhs = -divergence(z, P.spacing) / scale
    div_tol = scale * max(atol, rtol * np.linalg.norm(div_rhs.reshape(-1)))
    floor = 100 * np.finfo(np.float64).eps * max(norm_b, np.finfo(np.float64).tiny) * sum(1 / d for d in P.spacing)
    div_tol = max(div_tol, floor)
    initial_u = P.helmholtz(b, p)
    guess = P.pack(initial_u, scale / h * p)
    rhs = P.pack(b, np.zeros(P.shape)) - P.action(guess)
    tolerance = .5 * min(momentum_tol, h * div_tol)
    P.poisson_solves = P.cycles = 0
    correction, info = gmres(P.action, rhs, P.precondition, tolerance, restart, max_iterations)
    u, q = P.unpack(guess + correction)
    p = h / scale * (q - q.mean())
    momentum, div = P.metrics(u, p, b)
    if momentum > momentum_tol or div > div_tol:
        raise RuntimeError('CN FGMRES true residual rejected')
    info.update(poisson_solves=P.poisson_solves, cycles=P.cycles, momentum_residual=momentum,
                momentum_tolerance=momentum_tol, divergence_norm=div, divergence_tolerance=div_tol)
    return u, p, info
