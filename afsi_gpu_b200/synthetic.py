"""Seeded synthetic inputs of the benchmark configurations.

No datasets or meshes are read: the reference's gmsh-generated LV/valve meshes
cannot be regenerated offline, so procedural structures stand in for them.

* 2D: a closed ellipse of Lagrangian points with seeded radial jitter, point
  forces N(0,1), and a face velocity made of seeded Fourier modes.
* 3D: a truncated prolate-spheroid shell (long axis x) meshed from a structured
  (radial, polar, azimuthal) hexahedral grid.  Each hexahedron is split into
  five tetrahedra, alternating the two mirror-image splits in a checkerboard so
  that shared faces match; the longest edge is a face diagonal.  Edges get
  one shared midpoint each (straight-sided P2 elements, the ``promote_p1``
  construction of ``afsi_torch/tetrahedron.py:45-56``).  The shell is open at
  the base (x > centre) and has a small apical opening, so no element is
  degenerate at the pole.
"""
from math import pi
import numpy as np
import torch

# five-tet splits of the unit cube; vertex id = i + 2j + 4k
_EVEN = (0, 3, 5, 6)           # i+j+k even
_ODD = (1, 2, 4, 7)


def _split(central, other):
    tets = [central]
    for v in other:
        i, j, k = v & 1, (v >> 1) & 1, (v >> 2) & 1
        nbrs = [(1 - i) + 2 * j + 4 * k, i + 2 * (1 - j) + 4 * k, i + 2 * j + 4 * (1 - k)]
        tets.append((v, *nbrs))
    return tets


_SPLIT_A = _split(_EVEN, _ODD)
_SPLIT_B = _split(_ODD, _EVEN)
EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))


def promote_p1(X, cells):
    """One shared midpoint per unique edge (P1 -> straight-sided P2)."""
    pairs = np.sort(cells[:, EDGES].reshape(-1, 2), axis=1)
    unique, inverse = np.unique(pairs, axis=0, return_inverse=True)
    mid = X[unique].mean(axis=1)
    p2 = np.concatenate((cells, X.shape[0] + inverse.reshape(-1, 6)), axis=1)
    return np.concatenate((X, mid)), p2


def prolate_shell(nr=3, ntheta=40, nphi=64, *, center=(.5, .5, .5), inner=(.25, .15, .15), outer=(.32, .22, .22),
                  theta=(.12 * pi, .72 * pi)):
    """P1 tetrahedral shell: returns X (N,3) float64 and cells (E,4) int64.

    theta is the polar angle from the -x axis (apex at x<centre); the shell is
    truncated at theta[1] (open base) and opened at theta[0] (apex hole).
    """
    if nphi % 2:
        raise ValueError('nphi must be even for a conforming checkerboard split')
    s = np.linspace(0, 1, nr + 1)
    t = np.linspace(theta[0], theta[1], ntheta + 1)
    f = np.arange(nphi) * (2 * pi / nphi)
    S, Tt, F = np.meshgrid(s, t, f, indexing='ij')
    a = inner[0] + S * (outer[0] - inner[0])
    b = inner[1] + S * (outer[1] - inner[1])
    c = inner[2] + S * (outer[2] - inner[2])
    X = np.stack((center[0] - a * np.cos(Tt), center[1] + b * np.sin(Tt) * np.cos(F),
                  center[2] + c * np.sin(Tt) * np.sin(F)), -1).reshape(-1, 3)

    def vid(i, j, k):
        return (i * (ntheta + 1) + j) * nphi + (k % nphi)

    cells = []
    for i in range(nr):
        for j in range(ntheta):
            for k in range(nphi):
                corner = [vid(i + (v & 1), j + ((v >> 1) & 1), k + ((v >> 2) & 1)) for v in range(8)]
                split = _SPLIT_A if (i + j + k) % 2 == 0 else _SPLIT_B
                cells.extend([[corner[v] for v in tet] for tet in split])
    return X, np.asarray(cells, dtype=np.int64)


def p2_shell(nr=3, ntheta=40, nphi=64, **kw):
    X, cells = prolate_shell(nr, ntheta, nphi, **kw)
    return promote_p1(X, cells)


def ellipse_points(count=20000, *, center=(.5, .125), semi=(.3, .1), spacing=1 / 256, seed=0, dtype=np.float64):
    """Closed ellipse with radial jitter U(-0.2h, 0.2h)."""
    rng = np.random.default_rng(seed)
    t = np.arange(count) * (2 * pi / count)
    r = 1 + rng.uniform(-.2 * spacing, .2 * spacing, count) / np.hypot(semi[0] * np.cos(t), semi[1] * np.sin(t))
    pts = np.stack((center[0] + semi[0] * r * np.cos(t), center[1] + semi[1] * r * np.sin(t)), -1)
    return pts.astype(dtype)


def fourier_velocity2d(grid, modes=8, seed=0, dtype=torch.float64):
    """Sum of `modes` seeded Fourier modes on each face lattice."""
    rng = np.random.default_rng(seed)
    Lx, Ly = grid.lengths
    out = []
    for c in range(2):
        xy = grid.coordinates(c, dtype=torch.float64).numpy()
        u = np.zeros(xy.shape[:2])
        for _ in range(modes):
            kx, ky = rng.integers(1, 6, 2)
            amp, ph1, ph2 = rng.standard_normal(), rng.uniform(0, 2 * pi), rng.uniform(0, 2 * pi)
            u += amp * np.sin(2 * pi * kx * xy[..., 0] / Lx + ph1) * np.cos(pi * ky * xy[..., 1] / Ly + ph2)
        out.append(torch.as_tensor(u, dtype=dtype))
    return tuple(out)


def fourier_velocity3d(grid, modes=8, seed=0, dtype=torch.float64):
    rng = np.random.default_rng(seed)
    out = []
    for c in range(3):
        xyz = grid.coordinates(c, dtype=torch.float64).numpy()
        u = np.zeros(xyz.shape[:3])
        for _ in range(modes):
            k = rng.integers(1, 5, 3)
            amp, ph = rng.standard_normal(), rng.uniform(0, 2 * pi, 3)
            u += amp * np.prod([np.sin(2 * pi * k[a] * xyz[..., a] / grid.lengths[a] + ph[a]) for a in range(3)], 0)
        out.append(torch.as_tensor(u, dtype=dtype))
    return tuple(out)


def mean_free_normal(shape, seed=0, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    r = torch.randn(shape, generator=g, dtype=torch.float64)
    return (r - r.mean()).to(dtype)


def divergence_free_faces(grid, seed=0):
    """Seeded face field with zero discrete divergence and zero wall-normal
    flux: the discrete curl of random edge potentials that vanish on every
    boundary edge (each potential lives on the cell edges along its axis)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid.shape
    hx, hy, hz = grid.spacing
    pot = []
    for shape in ((nx, ny + 1, nz + 1), (nx + 1, ny, nz + 1), (nx + 1, ny + 1, nz)):
        a = rng.standard_normal(shape)
        for axis, n in enumerate(shape):
            if n != (nx, ny, nz)[axis]:  # node axes: clear both boundary planes
                a[(slice(None),) * axis + (0,)] = 0.
                a[(slice(None),) * axis + (n - 1,)] = 0.
        pot.append(a)
    ax, ay, az = pot
    u = np.diff(az, axis=1) / hy - np.diff(ay, axis=2) / hz
    v = np.diff(ax, axis=2) / hz - np.diff(az, axis=0) / hx
    w = np.diff(ay, axis=0) / hx - np.diff(ax, axis=1) / hy
    return tuple(torch.as_tensor(f) for f in (u, v, w))
