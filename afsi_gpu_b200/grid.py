"""Staggered (MAC) grid descriptions used by the transfers and solvers.

A grid here is an immutable description: cell counts per axis, the box
lengths, the lower corner, and the geometry derived from them once at
construction (spacing, cell volume, the shape and first-node position of each
face lattice).  Pressure lives at cell centres; velocity component c lives on
the faces normal to axis c, a lattice with one more node along c.  Arrays are
indexed (x, y[, z]) with the last axis fastest, the layout of the reference's
``MACGrid`` (``afsi_torch/mac/grid.py:13-59``) and ``ChannelGrid``
(``afsi_torch/mac2d/grid.py:7-43``), so tensors pass between the two without
copies.  Only the constructor signatures and attribute names follow the
reference; everything that consumes a grid in this package reads just
``shape``, ``lengths``, ``spacing``, ``volume``, ``face_shape`` and (3D)
``origin``/``face_origin``, so the reference's own grid objects are accepted
as they are.

``ChannelGrid(periodic=True)`` describes the same 2D lattices with a pressure
problem that wraps in x and has walls in y (no reference counterpart).
"""
from math import isfinite
import torch


def _cell_counts(values, dim, what):
    counts = tuple(values)
    if len(counts) != dim or not all(isinstance(n, int) and not isinstance(n, bool) and n >= 4 for n in counts):
        raise ValueError(f'{what}: {dim} integer cell counts, each at least 4, are required (got {values!r})')
    return counts


def _reals(values, dim, what, *, positive):
    out = tuple(float(v) for v in values)
    if len(out) != dim or not all(isfinite(v) and (v > 0 or not positive) for v in out):
        kind = 'positive finite' if positive else 'finite'
        raise ValueError(f'{what}: {dim} {kind} values are required (got {values!r})')
    return out


class _Staggered:
    """Geometry shared by the 2D and 3D staggered grids (dim set by the subclass)."""
    dim = 0
    __slots__ = ('shape', 'lengths', 'origin', 'spacing', 'volume', '_face_shapes', '_face_origins', '_key')

    def _setup(self, shape, lengths, origin, extra=()):
        put = object.__setattr__
        put(self, 'shape', _cell_counts(shape, self.dim, type(self).__name__ + ' shape'))
        put(self, 'lengths', _reals(lengths, self.dim, type(self).__name__ + ' lengths', positive=True))
        put(self, 'origin', _reals(origin, self.dim, type(self).__name__ + ' origin', positive=False))
        h = tuple(L / n for L, n in zip(self.lengths, self.shape))
        vol = 1.0
        for x in h:
            vol *= x
        put(self, 'spacing', h)
        put(self, 'volume', vol)
        eye = [[int(a == c) for a in range(self.dim)] for c in range(self.dim)]
        put(self, '_face_shapes', tuple(tuple(n + e for n, e in zip(self.shape, row)) for row in eye))
        # a face lattice sits on the cell walls along its own axis and at the
        # cell centres along the others
        put(self, '_face_origins', tuple(tuple(o + (1 - e) * .5 * d for o, d, e in zip(self.origin, h, row))
                                         for row in eye))
        put(self, '_key', (type(self).__name__, self.shape, self.lengths, self.origin) + tuple(extra))

    def __setattr__(self, name, value):
        raise AttributeError(f'{type(self).__name__} is immutable')

    def __eq__(self, other):
        return isinstance(other, _Staggered) and self._key == other._key

    def __hash__(self):
        return hash(self._key)

    def __repr__(self):
        return f'{type(self).__name__}(shape={self.shape}, lengths={self.lengths}, origin={self.origin})'

    # -- lattices
    def face_shape(self, component):
        return self._face_shapes[component]

    def face_origin(self, component):
        return self._face_origins[component]

    def cell_origin(self):
        """Position of the first cell centre."""
        return tuple(o + .5 * h for o, h in zip(self.origin, self.spacing))

    def coordinates(self, component=None, *, device='cpu', dtype=torch.float64):
        """Node positions of the pressure lattice (component None) or of a face
        lattice, shape ``lattice shape + (dim,)``."""
        if component is None:
            counts, first = self.shape, self.cell_origin()
        else:
            counts, first = self._face_shapes[component], self._face_origins[component]
        axes = [torch.arange(n, device=device, dtype=dtype).mul_(h).add_(o)
                for n, h, o in zip(counts, self.spacing, first)]
        return torch.stack(torch.meshgrid(*axes, indexing='ij'), dim=-1)

    def zeros(self, *, device='cpu', dtype=torch.float64):
        """One zero-filled array per velocity component."""
        return tuple(torch.zeros(s, device=device, dtype=dtype) for s in self._face_shapes)

    def check_velocity(self, velocity):
        """Raise ValueError unless `velocity` holds one floating array per
        component, on its face lattice, all of one dtype and device."""
        if len(velocity) != self.dim:
            raise ValueError(f'expected {self.dim} velocity components, got {len(velocity)}')
        first = velocity[0]
        for c, u in enumerate(velocity):
            if tuple(u.shape) != self._face_shapes[c]:
                raise ValueError(f'velocity component {c} has shape {tuple(u.shape)}, '
                                 f'expected {self._face_shapes[c]}')
            if u.dtype not in (torch.float32, torch.float64) or u.dtype != first.dtype or u.device != first.device:
                raise ValueError('velocity components must share one floating dtype and one device')


class MACGrid(_Staggered):
    """3D closed box: ``MACGrid(shape, lengths, origin=(0, 0, 0))``."""
    dim = 3
    __slots__ = ()

    def __init__(self, shape, lengths, origin=(0., 0., 0.)):
        self._setup(shape, lengths, origin)


class ChannelGrid(_Staggered):
    """2D channel with its lower-left corner at the origin:
    ``ChannelGrid(shape=(256, 64), lengths=(8, 1.61), periodic=False)``."""
    dim = 2
    __slots__ = ('periodic',)

    def __init__(self, shape=(256, 64), lengths=(8., 1.61), periodic=False):
        object.__setattr__(self, 'periodic', bool(periodic))
        self._setup(shape, lengths, (0., 0.), extra=(self.periodic,))

    def __repr__(self):
        return (f'ChannelGrid(shape={self.shape}, lengths={self.lengths}'
                + (', periodic=True)' if self.periodic else ')'))
