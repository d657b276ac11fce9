"""Adaptive interaction quadrature for P1 and P2 tetrahedra (host-side setup).

Small reference tables are built on the CPU once per order, as in the
reference.  The per-element orders, the comparison with the previous rule and
the order histogram come from one native launch (``afsi_b200_p2_orders``);
grouping cells, when the orders changed, runs as tensor ops on the device.
Follows ``afsi_torch/mac/adaptive_transfer.py:95-301``:

* Gaussian order per cell ``max(3, ceil(density * diam / dx_min))`` where diam
  is the diameter of the quadratic Bernstein hull of the P2 element
  (``:173-187``);
* ``conical`` rule family: Keast's positive degree-5 table for order 3
  (``p1.py:12-30``), otherwise the collapsed (Duffy) tensor product of
  Gauss–Jacobi rules with weights (1-u)^2, (1-v)^1, 1 (``:107-139``);
* one quadrature group per distinct order, points element-major.
"""
from dataclasses import dataclass
from itertools import permutations
from math import ceil
import numpy as np
import torch

# P2 local node order v0..v3, e01, e02, e03, e12, e13, e23 (tetrahedron.py:1-13)
EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))

# Keast degree-5 orbits (barycentric, weight); 15 points.
_KEAST5 = (((.25,) * 4, .030283678097089182),
           ((0., 1 / 3, 1 / 3, 1 / 3), .006026785714285717),
           ((8 / 11, 1 / 11, 1 / 11, 1 / 11), .011645249086028967),
           ((.4334498464263357, .4334498464263357, .0665501535736643, .0665501535736643), .010949141561386449))


def gauss_jacobi_unit(n, alpha):
    """n-point Gauss rule for ∫_0^1 f(u) (1-u)^alpha du (Golub–Welsch).

    Symmetric tridiagonal Jacobi matrix of the P^(alpha,0) recurrence on
    [-1,1], eigenvalues mapped to [0,1]; weights are the squared first
    eigenvector components times ∫_0^1 (1-u)^alpha du = 1/(alpha+1).
    """
    k = np.arange(n, dtype=float)
    d = 2 * k + alpha
    diag = np.zeros(n) if alpha == 0 else -alpha * alpha / (d * (d + 2))
    j = np.arange(1, n, dtype=float)
    a = 2 * j + alpha
    off = np.sqrt(4 * j * j * (j + alpha) ** 2 / (a * a * (a * a - 1)))
    nodes, vectors = np.linalg.eigh(np.diag(diag) + np.diag(off, 1) + np.diag(off, -1))
    return (nodes + 1) / 2, vectors[0] ** 2 / (alpha + 1)


def keast5():
    pts, wts = [], []
    for orbit, weight in _KEAST5:
        for bary in sorted(set(permutations(orbit))):
            pts.append(bary[1:])
            wts.append(weight)
    return np.asarray(pts), np.asarray(wts)


def conical_rule(order):
    """Positive degree ``2*order-1`` rule on the unit tetrahedron (points (Q,3), weights (Q,))."""
    if type(order) is not int or order < 2:
        raise ValueError('Gaussian order must be an integer >=2')
    if order == 3:
        return keast5()
    (u, a), (v, b), (w, c) = (gauss_jacobi_unit(order, al) for al in (2, 1, 0))
    U, V, Wn = np.meshgrid(u, v, w, indexing='ij')
    A, B, C = np.meshgrid(a, b, c, indexing='ij')
    pts = np.stack((U, (1 - U) * V, (1 - U) * (1 - V) * Wn), -1).reshape(-1, 3)
    return pts, (A * B * C).reshape(-1)


def tabulate_p2(points):
    """P2 Lagrange basis N[q,a] at reference points (tetrahedron.py:102-113)."""
    q = np.asarray(points, dtype=np.float64)
    L = np.concatenate((1 - q.sum(-1, keepdims=True), q), -1)
    i = np.array([e[0] for e in EDGES])
    j = np.array([e[1] for e in EDGES])
    return np.concatenate((L * (2 * L - 1), 4 * L[:, i] * L[:, j]), -1)


def reference_determinants(X, cells):
    """|det| of the reference edge matrix per cell (scalar triple product)."""
    v = X[cells[:, :4]]
    D = (v[:, 1:] - v[:, :1]).transpose(-1, -2)
    return (D[..., 0, :] * torch.linalg.cross(D[..., 1, :], D[..., 2, :])).sum(-1).abs()


@dataclass(frozen=True)
class QuadratureGroup:
    cells: torch.Tensor    # (E_g,10) int64
    values: torch.Tensor   # N (Q,10)
    weights: torch.Tensor  # W (E_g,Q) physical weights
    order: int = 0


@dataclass(frozen=True)
class InteractionRule:
    groups: tuple
    orders: torch.Tensor
    point_count: int


class RuleBuilder:
    """Caches reference tables per order and builds grouped rules
    (``AdaptiveFETransfer._rule``, ``mac/adaptive_transfer.py:266-301``)."""

    def __init__(self, X, cells, grid, *, point_density=2., max_order=8, max_points=12000000):
        from . import _lib
        _lib.require_cuda(X)
        if cells.dim() != 2 or cells.shape[1] not in (4, 10):
            raise ValueError('adaptive interaction rules need P1 (4-node) or P2 (10-node) tetrahedra')
        self.cells = cells
        self.p2 = cells.shape[1] == 10
        self.grid = grid
        self.density = float(point_density)
        self.max_order, self.max_points = max_order, max_points
        self.bins = max_order + 1
        self.min_order = 3 if self.p2 else 2   # _orders_p2 / _orders clamps (adaptive_transfer.py:167-187)
        self.determinants = reference_determinants(X, cells)
        self._tables = {}
        self._last = None

    @property
    def last(self):
        return self._last

    def tables(self, order, like):
        if order not in self._tables:
            q, w = conical_rule(order)
            N = tabulate_p2(q) if self.p2 else np.concatenate((1 - q.sum(-1, keepdims=True), q), -1)
            self._tables[order] = (torch.as_tensor(N, dtype=like.dtype, device=like.device),
                                   torch.as_tensor(w, dtype=like.dtype, device=like.device))
        return self._tables[order]

    def launch(self, x):
        """Queue the order kernel; nothing is read back.  Returns the orders and
        the int32 summary ``[changed, max, flags, hist[bins], spare]``; the
        spare slot can take the status word of a following prepare."""
        from . import _lib
        x = x.contiguous()
        E = self.cells.shape[0]
        orders = torch.empty(E, dtype=torch.int64, device=x.device)
        summary = torch.zeros(4 + self.bins, dtype=torch.int32, device=x.device)
        last = None if self._last is None else self._last.orders
        _lib.call('afsi_b200_p2_orders' if self.p2 else 'afsi_b200_p1_orders', _lib.ptr(x), x.shape[0],
                  _lib.ptr(self.cells), E, float(min(self.grid.spacing)), self.density, self.min_order,
                  _lib.ptr(orders),
                  None if last is None else _lib.ptr(last), _lib.ptr(summary), self.bins,
                  _lib.dtype_code(x.dtype), _lib.stream(x.device))
        return orders, summary

    def finish(self, x, orders, counts):
        """Rule for ``orders`` given the host copy ``counts`` of the summary."""
        from . import _lib
        changed, top, flags = counts[0], counts[1], counts[2]
        if flags & _lib.FLAG_INDEX:
            raise RuntimeError('P2 connectivity outside the node range')
        if flags & _lib.FLAG_SUPPORT:
            raise ValueError('MAC IB support reaches a wall or is nonfinite; enlarge/refine the fluid box')
        if self._last is not None and changed == 0:
            return self._last
        if top > self.max_order:
            raise ValueError(f'adaptive IB needs Gaussian order {top}, exceeds max_order={self.max_order}')
        hist = counts[3:3 + self.bins]
        groups, total = [], 0
        for n, count in enumerate(hist):
            if not count:
                continue
            N, w = self.tables(n, x)
            ids = torch.where(orders == n)[0]
            groups.append(QuadratureGroup(self.cells[ids].contiguous(), N,
                                          (self.determinants[ids, None] * w).contiguous(), n))
            total += count * len(w)
        if total > self.max_points:
            raise ValueError(f'adaptive IB needs {total} points, exceeds max_points={self.max_points}')
        self._last = InteractionRule(tuple(groups), orders, total)
        return self._last

    def __call__(self, x):
        orders, summary = self.launch(x)
        return self.finish(x, orders, summary.cpu().tolist())


def point_count_for(orders_histogram):
    return sum(count * (15 if n == 3 else n ** 3) for n, count in orders_histogram.items())


def order_for(diameter, dx, density=2.):
    return max(3, ceil(density * diameter / dx))
