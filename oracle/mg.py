"""NumPy restatement of the MAC geometric multigrid (oracle; test infrastructure only).

Three boundary conditions:

* ``neumann3d``: closed-box 3D pressure, ``mac/multigrid.py`` and
  ``mac/mg_workspace.py`` (mean-zero gauge, rank-one coarse fix).
* ``channel2d``: 2D inlet/outlet channel, ``mac2d/multigrid.py`` (Dirichlet
  outlet ghost, no gauge).
* ``dirichlet3d``: open box with zero pressure on the physical faces,
  ``mac/dirichlet_mg.py`` and ``mac/open_boundary.py`` (no gauge, odd
  extension in the prolongation).
* ``periodic2d``: periodic in x, no-slip (Neumann pressure) in y.  The
  reference has no such solver; this restatement follows the channel V-cycle
  structure (``mac2d/multigrid.py:56-82``) with the Neumann gauge and the
  rank-one coarse inverse of ``mac/multigrid.py:49-59``, x-wrapped stencils and
  periodic prolongation ghosts.

Jacobi weight 2/3, ``smooth`` sweeps before and after, restriction by child
averaging and cell-centred (bi/tri)linear prolongation (``align_corners=False``).
"""
from math import isfinite, prod
import numpy as np

OMEGA = 2 / 3


# ----------------------------------------------------------------- operators

def neg_laplacian3d(p, spacing):
    """``mac/grid.py:86-93``: per-axis ``out[:-1]-=d; out[1:]+=d``, d=diff/(h*h)."""
    out = np.zeros_like(p)
    for c, h in enumerate(spacing):
        d = np.diff(p, axis=c) / p.dtype.type(h * h)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[c] = slice(None, -1)
        hi[c] = slice(1, None)
        out[tuple(lo)] -= d
        out[tuple(hi)] += d
    return out


def diagonal3d(shape, spacing, dtype=np.float64):
    """``mac/multigrid.py:38-42``: ``+1/h**2`` per existing neighbour, axis order."""
    diag = np.zeros(shape, dtype=dtype)
    for c, h in enumerate(spacing):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[c] = slice(None, -1)
        hi[c] = slice(1, None)
        diag[tuple(lo)] += dtype(1 / h ** 2)
        diag[tuple(hi)] += dtype(1 / h ** 2)
    return diag


def neg_laplacian2d(p, spacing, bc):
    """Channel: ``mac2d/grid.py:61-71`` (outlet ``+2p/hx**2``).  Periodic: x
    differences wrap (every cell has both x neighbours), y one-sided rows.
    """
    hx, hy = spacing
    t = p.dtype.type
    out = np.zeros_like(p)
    if bc == 'channel':
        dx = (p[1:] - p[:-1]) / t(hx ** 2)
        out[:-1] -= dx
        out[1:] += dx
    else:
        dx = (np.roll(p, -1, 0) - p) / t(hx ** 2)      # d[i] = p[i+1]-p[i], wrapped
        out -= dx
        out += np.roll(dx, 1, 0)
    dy = (p[:, 1:] - p[:, :-1]) / t(hy ** 2)
    out[:, :-1] -= dy
    out[:, 1:] += dy
    if bc == 'channel':
        out[-1] += 2 * p[-1] / t(hx ** 2)
    return out


def diagonal2d(shape, spacing, bc, dtype=np.float64):
    """``mac2d/multigrid.py:26-33`` (channel); periodic: ``2/hx**2`` in x."""
    hx, hy = spacing
    diag = np.zeros(shape, dtype=dtype)
    if bc == 'channel':
        diag[:-1] += dtype(1 / hx ** 2)
        diag[1:] += dtype(1 / hx ** 2)
    else:
        diag += dtype(1 / hx ** 2)
        diag += dtype(1 / hx ** 2)
    diag[:, :-1] += dtype(1 / hy ** 2)
    diag[:, 1:] += dtype(1 / hy ** 2)
    if bc == 'channel':
        diag[-1] += dtype(2 / hx ** 2)
    return diag


def restrict3d(fine):
    """``F.avg_pool3d(.,2,2)`` / ``mac/_triton_mg.py:52-68``: 8 children summed
    x-major, z fastest, times 1/8."""
    n = tuple(s // 2 for s in fine.shape)
    v = None
    for a in range(2):
        for b in range(2):
            for c in range(2):
                child = fine[a::2, b::2, c::2][:n[0], :n[1], :n[2]]
                v = child.copy() if v is None else v + child
    return v * fine.dtype.type(.125)


def restrict2d(fine):
    """``mac2d/_triton_mg.py:41-52``: ``((r00+r01)+r10+r11)*.25``."""
    r00, r01 = fine[0::2, 0::2], fine[0::2, 1::2]
    r10, r11 = fine[1::2, 0::2], fine[1::2, 1::2]
    return ((r00 + r01) + r10 + r11) * fine.dtype.type(.25)


def neg_laplacian3d_dirichlet(p, spacing):
    """``mac/open_boundary.py:14-24``: -div(grad p) with the boundary-face
    gradient 2p/h (zero pressure half a cell outside), divergence summed over
    axes in order (``mac/grid.py:70-71``)."""
    out = None
    for c, h in enumerate(spacing):
        t = p.dtype.type(h)
        first = [slice(None)] * 3
        last = [slice(None)] * 3
        first[c] = slice(0, 1)
        last[c] = slice(-1, None)
        g = np.concatenate((2 * p[tuple(first)] / t, np.diff(p, axis=c) / t, -2 * p[tuple(last)] / t), c)
        d = np.diff(g, axis=c) / t
        out = d if out is None else out + d
    return -out


def diagonal3d_dirichlet(shape, spacing, dtype=np.float64):
    """``mac/open_boundary.py:47-52``: 2·Σh⁻² plus h⁻² on each boundary face."""
    diag = np.full(shape, 2 * sum(h ** -2 for h in spacing), dtype=dtype)
    for c, h in enumerate(spacing):
        first = [slice(None)] * 3
        last = [slice(None)] * 3
        first[c] = slice(0, 1)
        last[c] = slice(-1, None)
        diag[tuple(first)] += dtype(h ** -2)
        diag[tuple(last)] += dtype(h ** -2)
    return diag


def prolong3d_dirichlet(coarse):
    """Odd extension by one ghost cell per side and axis, trilinear 2x
    (``align_corners=False``), cropped to the interior
    (``mac/dirichlet_mg.py:52-62``): fine i reads padded coarse i/2+3/4."""
    padded = coarse
    for c in range(3):
        first = [slice(None)] * 3
        last = [slice(None)] * 3
        first[c] = slice(0, 1)
        last[c] = slice(-1, None)
        padded = np.concatenate((-padded[tuple(first)], padded, -padded[tuple(last)]), c)
    def axis(n):
        i = np.arange(n)
        src = i / 2 + .75
        i0 = np.floor(src).astype(np.int64)
        l1 = src - i0
        return i0, i0 + 1, 1 - l1, l1
    dt = coarse.dtype
    x0, x1, wx0, wx1 = axis(2 * coarse.shape[0])
    y0, y1, wy0, wy1 = axis(2 * coarse.shape[1])
    z0, z1, wz0, wz1 = axis(2 * coarse.shape[2])
    wx0, wx1, wy0, wy1, wz0, wz1 = (w.astype(dt) for w in (wx0, wx1, wy0, wy1, wz0, wz1))
    cz = padded[:, :, z0] * wz0 + padded[:, :, z1] * wz1
    cy = cz[:, y0, :] * wy0[:, None] + cz[:, y1, :] * wy1[:, None]
    return cy[x0] * wx0[:, None, None] + cy[x1] * wx1[:, None, None]


def _axis_weights(n_fine, n_coarse):
    """Source index/weights of ``F.interpolate(..., align_corners=False)`` for 2x:
    ``src=max((i+.5)/2-.5,0)``, ``i1=i0+(i0<n-1)``."""
    i = np.arange(n_fine)
    src = np.maximum((i + .5) * (n_coarse / n_fine) - .5, 0.)
    i0 = np.floor(src).astype(np.int64)
    i1 = np.minimum(i0 + 1, n_coarse - 1)
    l1 = src - i0
    return i0, i1, 1 - l1, l1


def prolong3d(coarse, fine_shape):
    """Trilinear, ``align_corners=False``, edge clamp (``mac/multigrid.py:121-122``)."""
    ix0, ix1, wx0, wx1 = _axis_weights(fine_shape[0], coarse.shape[0])
    iy0, iy1, wy0, wy1 = _axis_weights(fine_shape[1], coarse.shape[1])
    iz0, iz1, wz0, wz1 = _axis_weights(fine_shape[2], coarse.shape[2])
    t = coarse.dtype.type
    wx0, wx1, wy0, wy1, wz0, wz1 = (w.astype(coarse.dtype) for w in (wx0, wx1, wy0, wy1, wz0, wz1))
    cz = coarse[:, :, iz0] * wz0 + coarse[:, :, iz1] * wz1
    cy = cz[:, iy0, :] * wy0[:, None] + cz[:, iy1, :] * wy1[:, None]
    return (cy[ix0] * wx0[:, None, None] + cy[ix1] * wx1[:, None, None]).astype(t)


def prolong2d(coarse, bc):
    """Bilinear with boundary ghosts, ``mac2d/multigrid.py:76-82``.

    Channel: even ghosts left/top/bottom, odd ghost at the outlet.  Periodic:
    x ghosts wrap, even in y.  Fine i maps to coarse ``i/2-1/4``.
    """
    if bc == 'channel':
        padded = np.concatenate((coarse[:1], coarse, -coarse[-1:]), 0)
    else:
        padded = np.concatenate((coarse[-1:], coarse, coarse[:1]), 0)
    padded = np.concatenate((padded[:, :1], padded, padded[:, -1:]), 1)
    nx, ny = 2 * coarse.shape[0], 2 * coarse.shape[1]
    # padded-grid source coordinate of fine i is i/2+.75
    def axis(n):
        i = np.arange(n)
        src = i / 2 + .75
        i0 = np.floor(src).astype(np.int64)
        l1 = src - i0
        return i0, i0 + 1, 1 - l1, l1
    x0, x1, wx0, wx1 = axis(nx)
    y0, y1, wy0, wy1 = axis(ny)
    dt = coarse.dtype
    wy0, wy1, wx0, wx1 = (w.astype(dt) for w in (wy0, wy1, wx0, wx1))
    cy = padded[:, y0] * wy0 + padded[:, y1] * wy1
    return cy[x0] * wx0[:, None] + cy[x1] * wx1[:, None]


# ------------------------------------------------------------------ hierarchy

class Hierarchy:
    """Levels, diagonals and the dense coarsest inverse.

    ``mac/multigrid.py:33-59`` (3D) / ``mac2d/multigrid.py:22-46`` (2D):
    halve while ``min(shape)>4`` and every extent is even; coarsest <= 512.
    """

    def __init__(self, shape, spacing, bc, dtype=np.float64, coarse_dtype=None):
        self.bc, self.dtype = bc, dtype
        self.dim = len(shape)
        self.shapes, self.spacings, self.diagonals = [], [], []
        shape, spacing = tuple(shape), tuple(spacing)
        while True:
            self.shapes.append(shape)
            self.spacings.append(spacing)
            if bc == 'dirichlet':
                self.diagonals.append(diagonal3d_dirichlet(shape, spacing, dtype))
            else:
                self.diagonals.append(diagonal3d(shape, spacing, dtype) if self.dim == 3
                                      else diagonal2d(shape, spacing, bc, dtype))
            if min(shape) <= 4 or any(n % 2 for n in shape):
                break
            shape = tuple(n // 2 for n in shape)
            spacing = tuple(2 * h for h in spacing)
        count = prod(shape)
        if count > 512:
            raise ValueError('MAC dimensions must coarsen to <=512 cells')
        cd = coarse_dtype or dtype
        eye = np.eye(count, dtype=np.float64)
        A = np.stack([self.apply(len(self.shapes) - 1, v.reshape(shape).astype(np.float64)).reshape(-1)
                      for v in eye], 1)
        if self.singular:
            A = A + np.ones_like(A) / count
        self.coarse_inverse = np.linalg.inv(A).astype(cd)

    @property
    def singular(self):
        return self.bc in ('neumann', 'periodic')

    def apply(self, level, p):
        h = self.spacings[level]
        if self.bc == 'dirichlet':
            return neg_laplacian3d_dirichlet(p, h)
        return neg_laplacian3d(p, h) if self.dim == 3 else neg_laplacian2d(p, h, self.bc)

    def restrict(self, r):
        return restrict3d(r) if self.dim == 3 else restrict2d(r)

    def prolong(self, coarse, shape):
        if self.bc == 'dirichlet':
            return prolong3d_dirichlet(coarse)
        return prolong3d(coarse, shape) if self.dim == 3 else prolong2d(coarse, self.bc)


def smooth(h, level, p, rhs, sweeps):
    """Weighted Jacobi, ``p+(2/3)*(rhs-Ap)/diag`` (``mac/multigrid.py:107-110``),
    then ``p-=mean`` for singular problems (``mac/mg_workspace.py:74-83``)."""
    w = h.dtype(OMEGA)
    for _ in range(sweeps):
        p = p + w * (rhs - h.apply(level, p)) / h.diagonals[level]
    if h.singular:
        p = p - p.mean(dtype=np.float64).astype(h.dtype)
    return p


def rb_smooth(h, level, p, rhs, sweeps):
    """Red-black Gauss-Seidel sweeps (the selectable smoother of the B200
    build; the reference has none): cells with an even index sum, then the
    odd ones, p += (rhs - A p)/diag in place (omega 1)."""
    color = np.indices(p.shape).sum(0) & 1
    d = h.diagonals[level]
    for _ in range(sweeps):
        for c in (0, 1):
            p = np.where(color == c, p + (rhs - h.apply(level, p)) / d, p)
    return p


def cycle(h, level, p, rhs, sweeps, smoother='jacobi'):
    """One V-cycle: ``mac/multigrid.py:112-123`` / ``mac2d/multigrid.py:67-83``.

    ``smoother='red-black'`` replaces the weighted Jacobi sweeps (and their
    per-sweep mean gauge) by red-black Gauss-Seidel sweeps; singular problems
    then shift the finest iterate to mean zero once, at the end of the cycle.
    """
    if smoother == 'red-black':
        p = _rb_cycle(h, level, p, rhs, sweeps)
        if level == 0 and h.singular:
            p = p - p.mean(dtype=np.float64).astype(h.dtype)
        return p
    if level == len(h.shapes) - 1:
        sol = (h.coarse_inverse.astype(np.float64) @ rhs.reshape(-1).astype(np.float64))
        sol = sol.astype(h.dtype).reshape(rhs.shape)
        if h.singular:
            sol = sol - sol.mean(dtype=np.float64).astype(h.dtype)
        return sol
    p = smooth(h, level, p, rhs, sweeps) if h.singular else _plain_smooth(h, level, p, rhs, sweeps)
    coarse = h.restrict(rhs - h.apply(level, p))
    if h.singular:
        coarse = coarse - coarse.mean(dtype=np.float64).astype(h.dtype)
    corr = cycle(h, level + 1, np.zeros_like(coarse), coarse, sweeps)
    p = p + h.prolong(corr, p.shape)
    return smooth(h, level, p, rhs, sweeps) if h.singular else _plain_smooth(h, level, p, rhs, sweeps)


def _rb_cycle(h, level, p, rhs, sweeps):
    if level == len(h.shapes) - 1:
        sol = (h.coarse_inverse.astype(np.float64) @ rhs.reshape(-1).astype(np.float64))
        sol = sol.astype(h.dtype).reshape(rhs.shape)
        if h.singular:
            sol = sol - sol.mean(dtype=np.float64).astype(h.dtype)
        return sol
    p = rb_smooth(h, level, p, rhs, sweeps)
    coarse = h.restrict(rhs - h.apply(level, p))
    if h.singular:
        coarse = coarse - coarse.mean(dtype=np.float64).astype(h.dtype)
    corr = _rb_cycle(h, level + 1, np.zeros_like(coarse), coarse, sweeps)
    p = p + h.prolong(corr, p.shape)
    return rb_smooth(h, level, p, rhs, sweeps)


def _plain_smooth(h, level, p, rhs, sweeps):
    w = h.dtype(OMEGA)
    for _ in range(sweeps):
        p = p + w * (rhs - h.apply(level, p)) / h.diagonals[level]
    return p


def solve(h, rhs, initial=None, *, rtol=1e-10, atol=1e-12, max_cycles=100, sweeps=4, check_every=2,
          smoother='jacobi'):
    """Solve loop, ``mac/multigrid.py:125-172`` (singular) and
    ``mac2d/multigrid.py:85-111`` (channel).  Returns (p, info)."""
    rhs = np.asarray(rhs, dtype=h.dtype)
    if not np.isfinite(rhs).all():
        raise ValueError('invalid pressure RHS')
    if h.singular:
        mean, amean = rhs.mean(dtype=np.float64), np.abs(rhs).mean(dtype=np.float64)
        if abs(mean) > 1e-12 + 1e-10 * amean:
            raise ValueError('incompatible Neumann pressure RHS: net flux must vanish')
        rhs = rhs - rhs.mean(dtype=np.float64).astype(h.dtype)
    p = np.zeros_like(rhs) if initial is None else np.array(initial, dtype=h.dtype)
    if h.singular:
        p = p - p.mean(dtype=np.float64).astype(h.dtype)
    rhs_norm = float(np.linalg.norm(rhs.astype(np.float64)))
    res = float(np.linalg.norm((rhs - h.apply(0, p)).astype(np.float64)))
    tol = max(atol, rtol * rhs_norm)
    if res <= tol:
        return p, dict(cycles=0, residual_norm=res, tolerance=tol)
    for k in range(1, max_cycles + 1):
        p = cycle(h, 0, p, rhs, sweeps, smoother)
        if k % check_every == 0 or k == max_cycles:
            res = float(np.linalg.norm((rhs - h.apply(0, p)).astype(np.float64)))
            if not isfinite(res):
                raise RuntimeError('nonfinite multigrid residual')
            if res <= tol:
                return p, dict(cycles=k, residual_norm=res, tolerance=tol)
    raise RuntimeError(f'multigrid did not converge: {res:g} > {tol:g}')
