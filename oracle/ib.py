"""NumPy restatement of the IB_4 transfers (oracle; test infrastructure only).

Covers the Peskin kernel, binning/prepare in its three table layouts, the
compact separable 3D spread/gather, the 2D reflected indexed transfer and the
P2 fused spread / gather-assemble.  Citations are afsi-torch 0.28.0 paths
relative to ``src/afsi_torch``.
"""
import numpy as np


def peskin4(distance):
    """Clamped two-branch IB_4 kernel, ``ib.py:57-67``.

    Same operation order as the torch expression: ``a=min(r,1)``,
    ``b=clip(r,1,2)``; inner ``((3-2a)+sqrt((1+4a)-4a^2))/8``; outer
    ``((5-2b)-sqrt((-7+12b)-4b^2))/8``; zero for ``r>=2``.
    """
    d = np.asarray(distance)
    r = np.abs(d)
    one, two = d.dtype.type(1), d.dtype.type(2)
    a = np.minimum(r, one)
    b = np.clip(r, one, two)
    inner = (3 - 2 * a + np.sqrt(1 + 4 * a - 4 * (a * a))) / 8
    outer = (5 - 2 * b - np.sqrt(-7 + 12 * b - 4 * (b * b))) / 8
    return np.where(r < 1, inner, np.where(r < 2, outer, np.zeros_like(r)))


def peskin4_radical(f):
    """Shared-radical form of the four weights for fractional offset ``f``.

    ``mac/csrc/p2_transfer.cu:36-43`` and ``mac/_triton_prepare.py:38-48``:
    ``r=sqrt((1+4f)-4(f*f))``, weights ``((3-2f)-r)/8, ((3-2f)+r)/8,
    ((1+2f)+r)/8, ((1+2f)-r)/8``.  Returns (..., 4).
    """
    f = np.asarray(f)
    rad = np.sqrt(1 + 4 * f - 4 * (f * f))
    return np.stack(((3 - 2 * f - rad) / 8, (3 - 2 * f + rad) / 8,
                     (1 + 2 * f + rad) / 8, (1 + 2 * f - rad) / 8), -1)


def compact_prepare(points, origins, spacing, form='clamped'):
    """Binning + 1D weights for L lattices, ``mac/compact_transfer.py:21-26``.

    points (P,3), origins (L,3), spacing (3,) -> base (L,P,3) int64,
    phi (L,P,3,4).  ``scaled=(x-o)/h``, ``base=floor(scaled-1)`` and either
    the clamped kernel on ``scaled-(base+k)`` (reference torch path) or the
    shared radical on ``f=scaled-base-1`` (reference CUDA/Triton path).
    """
    points = np.asarray(points)
    dt = points.dtype.type
    origins = np.asarray(origins, dtype=points.dtype)
    spacing = np.asarray(spacing, dtype=points.dtype)
    scaled = (points[None] - origins[:, None]) / spacing
    base = np.floor(scaled - dt(1)).astype(np.int64)
    if form == 'clamped':
        nodes = base[..., None] + np.arange(4)
        phi = peskin4(scaled[..., None] - nodes.astype(points.dtype))
    elif form == 'radical':
        f = scaled - base.astype(points.dtype) - dt(1)
        phi = peskin4_radical(f)
    else:
        raise ValueError(form)
    return base, phi


def shared_origins(origin, spacing, dtype=np.float64):
    """Face lattice at ``origin`` and centre lattice at ``origin+h/2``.

    ``mac/adaptive_transfer.py:225-229`` (shared stencil origins).
    """
    o = np.asarray(origin, dtype=np.float64)
    h = np.asarray(spacing, dtype=np.float64)
    return np.stack((o, o + .5 * h)).astype(dtype)


def face_origins(origin, spacing, dtype=np.float64):
    """Component face origins, ``mac/grid.py:38-40``."""
    rows = []
    for c in range(3):
        rows.append([o + (0. if a == c else .5 * h) for a, (o, h) in enumerate(zip(origin, spacing))])
    return np.asarray(rows, dtype=dtype)


def expand_shared(base, phi):
    """Shared (2,P,3) tables -> per-component (3,P,3) tables.

    ``mac/shared_stencil.py:13-19``: component c reads the face lattice along
    axis c and the centre lattice along the other axes.
    """
    b = np.stack([np.stack([base[int(a != c), :, a] for a in range(3)], -1) for c in range(3)])
    p = np.stack([np.stack([phi[int(a != c), :, a, :] for a in range(3)], 1) for c in range(3)])
    return b, p


def _links(base, phi, shape):
    """Expanded 64 links of one component, ``compact_transfer.py:133-140``.

    z fastest, then y, then x; weight ``(phi_x*phi_y)*phi_z``.
    """
    nodes = base[..., None] + np.arange(4)
    ids = ((nodes[:, 0, :, None, None] * shape[1] + nodes[:, 1, None, :, None])
           * shape[2] + nodes[:, 2, None, None, :])
    w = (phi[:, 0, :, None, None] * phi[:, 1, None, :, None]) * phi[:, 2, None, None, :]
    return ids.reshape(-1, 64), w.reshape(-1, 64)


def compact_spread(force, base, phi, shape, volume, chunk=65536):
    """One component of ``compact_spread``: ``mac/csrc/transfer.cu:33-53`` and
    ``compact_transfer.py:150-163`` (contribution ``(w*f)/volume``).
    """
    n = int(np.prod(shape))
    out = np.zeros(n, dtype=force.dtype)
    for s in range(0, len(force), chunk):
        ids, w = _links(base[s:s + chunk], phi[s:s + chunk], shape)
        out += np.bincount(ids.reshape(-1), weights=((w * force[s:s + chunk, None]) / volume).reshape(-1),
                           minlength=n).astype(force.dtype)
    return out


def compact_gather(field, base, phi, shape, chunk=65536):
    """One component of ``compact_gather``: ``Σ_links u[id]*w``,
    ``mac/csrc/transfer.cu:33-53`` and ``compact_transfer.py:165-179``.
    """
    flat = np.asarray(field).reshape(-1)
    out = np.empty(len(base), dtype=flat.dtype)
    for s in range(0, len(base), chunk):
        ids, w = _links(base[s:s + chunk], phi[s:s + chunk], shape)
        out[s:s + chunk] = (flat[ids] * w).sum(-1)
    return out


def grid_face_shape(shape, c):
    """``mac/grid.py:35-36`` / ``mac2d/grid.py:26-27``."""
    return tuple(n + (a == c) for a, n in enumerate(shape))


def spread3d(force, base3, phi3, shape, volume):
    """All three components from per-component tables (3,P,3)/(3,P,3,4)."""
    return tuple(compact_spread(np.ascontiguousarray(force[:, c]), base3[c], phi3[c],
                                grid_face_shape(shape, c), volume) for c in range(3))


def gather3d(fields, base3, phi3, shape):
    return np.stack([compact_gather(fields[c], base3[c], phi3[c], grid_face_shape(shape, c))
                     for c in range(3)], -1)


def support_valid3d(points, origin, spacing, shape):
    """``compact_transfer.py:94-96``: finite and ``2 <= (x-o)/h < n-2``."""
    points = np.asarray(points)
    scaled = (points - np.asarray(origin, points.dtype)) / np.asarray(spacing, points.dtype)
    limits = np.asarray(shape, points.dtype) - 2
    return bool(np.isfinite(points).all() and (scaled >= 2).all() and (scaled < limits).all())


# --------------------------------------------------------------------------- 2D

def prepare2d(points, shape, spacing):
    """Reflected 4x4 channel stencils, ``mac2d/transfer.py:61-81``.

    points (P,2) -> ids (2,P,16) int64, weights (2,P,16).  Offsets are
    ``(i,j)`` with j fastest; rows outside the wall are reflected (u: ``-j-1``
    / ``2ny-j-1``; v: ``-j`` / ``2ny-j``) and their weight negated.
    """
    points = np.asarray(points)
    dt = points.dtype.type
    h = np.asarray(spacing, dtype=points.dtype)
    ny = shape[1]
    offs = np.stack(np.meshgrid(np.arange(4), np.arange(4), indexing='ij'), -1).reshape(16, 2)
    ids, ws = [], []
    for c in range(2):
        origin = h * np.asarray([0 if c == 0 else .5, 0 if c == 1 else .5], dtype=points.dtype)
        scaled = (points - origin) / h
        nodes = np.floor(scaled - dt(1)).astype(np.int64)[:, None] + offs[None]
        w = peskin4(scaled[:, None] - nodes.astype(points.dtype))
        w = w[..., 0] * w[..., 1]
        j = nodes[..., 1]
        if c == 0:
            outside = (j < 0) | (j >= ny)
            refl = np.where(j < 0, -j - 1, np.where(j >= ny, 2 * ny - j - 1, j))
        else:
            outside = (j < 0) | (j > ny)
            refl = np.where(j < 0, -j, np.where(j > ny, 2 * ny - j, j))
        w = np.where(outside, -w, w)
        fs = grid_face_shape(shape, c)
        ids.append(nodes[..., 0] * fs[1] + refl)
        ws.append(w)
    return np.stack(ids), np.stack(ws)


def support_valid2d(points, lengths, spacing):
    """``mac2d/transfer.py:97-101``."""
    hx, hy = spacing
    p = np.asarray(points)
    return bool(np.isfinite(p).all() and (p[:, 0] >= 2 * hx).all() and (p[:, 0] <= lengths[0] - 2 * hx).all()
                and (p[:, 1] >= -hy).all() and (p[:, 1] <= lengths[1] + hy).all())


def indexed_spread(force, ids, weights, size, volume):
    """``mac/csrc/transfer.cu:10-29`` spread / ``mac2d/transfer.py:113-115``:
    ``out[ids] += (f*w)/volume`` for one component column ``force`` (P,).
    """
    contrib = (force[:, None] * weights) / volume
    return np.bincount(ids.reshape(-1), weights=contrib.reshape(-1), minlength=size).astype(force.dtype)


def indexed_gather(field, ids, weights):
    """``mac/csrc/transfer.cu:10-29`` gather / ``mac2d/transfer.py:127``."""
    return (np.asarray(field).reshape(-1)[ids] * weights).sum(-1)


# --------------------------------------------------------------------------- P2

def p2_points(x, cells, N):
    """x_q = Σ_a N[q,a]*x[cell_a], summed a=0..9 in order without FMA.

    ``mac/csrc/p2_transfer.cu:19-27``.  Returns (E*Q,3), element-major.
    """
    x = np.asarray(x)
    pos = np.zeros((cells.shape[0], N.shape[0], 3), dtype=x.dtype)
    for a in range(cells.shape[1]):
        pos = pos + N[None, :, a, None] * x[cells[:, a]][:, None, :]
    return pos.reshape(-1, 3)


def p2_prepare(x, groups, origin, spacing, shape):
    """Shared face/centre tables for all groups, ``mac/csrc/p2_transfer.cu:12-45``
    and ``mac/p2_cuda_transfer.py:18-39``.

    groups: list of (cells (E,10), N (Q,10)).  Returns base (2,T,3), phi
    (2,T,3,4), invalid flag.  Invalid points (outside ``2 <= s < n-2``) get
    ``scaled=0`` tables, as in the reference kernel.
    """
    x = np.asarray(x)
    dt = x.dtype.type
    o = np.asarray(origin, dtype=x.dtype)
    h = np.asarray(spacing, dtype=x.dtype)
    limits = np.asarray(shape, dtype=x.dtype) - dt(2)
    pts = np.concatenate([p2_points(x, c, N) for c, N in groups])
    physical = (pts - o) / h
    valid = np.isfinite(physical) & (physical >= 2) & (physical < limits)
    bases, phis = [], []
    for lattice in range(2):
        start = o + dt(.5) * h if lattice else o
        scaled = np.where(valid, (pts - start) / h, dt(0))
        lower = np.floor(scaled - dt(1)).astype(np.int64)
        f = scaled - lower.astype(x.dtype) - dt(1)
        bases.append(lower)
        phis.append(peskin4_radical(f))
    return np.stack(bases), np.stack(phis), int(not valid.all())


def p2_weighted_force(coef, cells, N, W):
    """F_q = (Σ_a N[q,a] coef[cell_a]) * W[e,q], ``mac/compact_transfer.py:29-35``."""
    val = np.zeros((cells.shape[0], N.shape[0], coef.shape[1]), dtype=coef.dtype)
    for a in range(cells.shape[1]):
        val = val + N[None, :, a, None] * coef[cells[:, a]][:, None, :]
    return (val * W[..., None]).reshape(-1, coef.shape[1])


def p2_assemble(U, cells, N, W, nodes):
    """rhs[cell_a] += Σ_q (N[q,a]*W[e,q])*U_q, ``mac/compact_transfer.py:37-39``."""
    E, Q = W.shape
    U = U.reshape(E, Q, -1)
    local = np.zeros((E, cells.shape[1], U.shape[-1]), dtype=U.dtype)
    for q in range(Q):
        local = local + (N[q][None, :] * W[:, q, None])[..., None] * U[:, q, None, :]
    out = np.zeros((nodes, U.shape[-1]), dtype=U.dtype)
    for c in range(U.shape[-1]):
        out[:, c] = np.bincount(cells.reshape(-1), weights=local[..., c].reshape(-1), minlength=nodes)
    return out


def p2_spread(coef, groups, base, phi, shape, volume):
    """``p2_spread_`` semantics (``mac/csrc/p2_transfer.cu:98-188``, Spread):
    weighted point forces of every group, spread with the shared tables.
    groups: list of (cells, N, W).
    """
    force = np.concatenate([p2_weighted_force(coef, c, N, W) for c, N, W in groups])
    b3, p3 = expand_shared(base, phi)
    return spread3d(force, b3, p3, shape, volume)


def p2_gather_assemble(fields, groups, base, phi, shape, nodes):
    """``p2_gather_assemble_`` semantics (``p2_transfer.cu:98-188``, Gather)."""
    b3, p3 = expand_shared(base, phi)
    U = gather3d(fields, b3, p3, shape)
    rhs = np.zeros((nodes, 3), dtype=U.dtype)
    off = 0
    for c, N, W in groups:
        n = W.size
        rhs += p2_assemble(U[off:off + n], c, N, W, nodes)
        off += n
    return rhs


TET_EDGES = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]])


def p2_orders(x, cells, dx, density, min_order=3):
    """Adaptive quadrature order of each P2 element, ``_orders_p2`` in
    ``mac/adaptive_transfer.py:173-187``: the Bernstein control points are the
    four corners and ``2 x_mid - (x_i + x_j)/2`` per edge; the order is
    ``ceil(density * diameter / dx)`` clamped below at 3."""
    nodes = np.asarray(x)[np.asarray(cells)]
    controls = 2 * nodes[:, 4:] - .5 * (nodes[:, TET_EDGES[:, 0]] + nodes[:, TET_EDGES[:, 1]])
    hull = np.concatenate((nodes[:, :4], controls), 1)
    a, b = np.triu_indices(10, 1)
    d = hull[:, a] - hull[:, b]
    squared = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    diameter = np.sqrt(squared.max(-1))
    return np.maximum(np.ceil(density * diameter / dx), min_order).astype(np.int64)


def p1_orders(x, cells, dx, density, min_order=2):
    """P1 element order, ``_orders`` in ``mac/adaptive_transfer.py:167-170``:
    ``ceil(density * longest_edge / dx)`` clamped below at 2."""
    nodes = np.asarray(x)[np.asarray(cells)]
    d = nodes[:, TET_EDGES[:, 0]] - nodes[:, TET_EDGES[:, 1]]
    squared = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    return np.maximum(np.ceil(density * np.sqrt(squared.max(-1)) / dx), min_order).astype(np.int64)
