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
