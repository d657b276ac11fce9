"""Staggered MAC grids with the reference's fields and layout.

``MACGrid`` follows ``afsi_torch/mac/grid.py:13-59`` (3D closed box, (x,y,z)
order, z fastest) and ``ChannelGrid`` follows ``afsi_torch/mac2d/grid.py:7-43``
(2D, y fastest).  ``ChannelGrid(periodic=True)`` is the same staggered layout
with a pressure operator that is periodic in x and has Neumann walls in y.
"""
from dataclasses import dataclass
from math import isfinite, prod
import torch


@dataclass(frozen=True)
class MACGrid:
    shape: tuple
    lengths: tuple
    origin: tuple = (0., 0., 0.)

    def __post_init__(self):
        if len(self.shape) != 3 or any(type(n) is not int or n < 4 for n in self.shape):
            raise ValueError('MAC requires three integer cell counts >= 4')
        if (len(self.lengths) != 3 or len(self.origin) != 3 or
                any(not isfinite(v) or v <= 0 for v in self.lengths) or
                any(not isfinite(v) for v in self.origin)):
            raise ValueError('finite origin and positive box lengths required')

    @property
    def spacing(self):
        return tuple(L / n for L, n in zip(self.lengths, self.shape))

    @property
    def volume(self):
        return prod(self.spacing)

    def face_shape(self, component):
        return tuple(n + (axis == component) for axis, n in enumerate(self.shape))

    def face_origin(self, component):
        return tuple(o + (0. if axis == component else .5 * h)
                     for axis, (o, h) in enumerate(zip(self.origin, self.spacing)))

    def zeros(self, *, device='cpu', dtype=torch.float64):
        return tuple(torch.zeros(self.face_shape(c), device=device, dtype=dtype) for c in range(3))

    def coordinates(self, component=None, *, device='cpu', dtype=torch.float64):
        shape = self.shape if component is None else self.face_shape(component)
        origin = (tuple(o + .5 * h for o, h in zip(self.origin, self.spacing))
                  if component is None else self.face_origin(component))
        axes = [o + h * torch.arange(n, device=device, dtype=dtype)
                for n, h, o in zip(shape, self.spacing, origin)]
        return torch.stack(torch.meshgrid(*axes, indexing='ij'), -1)

    def check_velocity(self, velocity):
        if len(velocity) != 3:
            raise ValueError('three MAC velocity components required')
        for c, u in enumerate(velocity):
            if (u.shape != self.face_shape(c) or u.dtype not in (torch.float32, torch.float64)
                    or u.device != velocity[0].device or u.dtype != velocity[0].dtype):
                raise ValueError('MAC field shape/device/dtype mismatch')


@dataclass(frozen=True)
class ChannelGrid:
    shape: tuple = (256, 64)
    lengths: tuple = (8., 1.61)
    periodic: bool = False

    def __post_init__(self):
        if len(self.shape) != 2 or any(type(n) is not int or n < 4 for n in self.shape):
            raise ValueError('two integer cell counts >=4 required')
        if len(self.lengths) != 2 or any(not isfinite(v) or v <= 0 for v in self.lengths):
            raise ValueError('two finite positive channel lengths required')

    @property
    def spacing(self):
        return tuple(L / n for L, n in zip(self.lengths, self.shape))

    @property
    def volume(self):
        return prod(self.spacing)

    def face_shape(self, c):
        return tuple(n + (axis == c) for axis, n in enumerate(self.shape))

    def coordinates(self, c=None, *, device='cpu', dtype=torch.float64):
        shape = self.shape if c is None else self.face_shape(c)
        axes = [h * (torch.arange(n, device=device, dtype=dtype) + (0 if c == a else .5))
                for a, (n, h) in enumerate(zip(shape, self.spacing))]
        return torch.stack(torch.meshgrid(*axes, indexing='ij'), -1)

    def zeros(self, *, device='cpu', dtype=torch.float64):
        return tuple(torch.zeros(self.face_shape(c), device=device, dtype=dtype) for c in range(2))

    def check_velocity(self, velocity):
        if len(velocity) != 2:
            raise ValueError('two velocity components required')
        for c, u in enumerate(velocity):
            if u.shape != self.face_shape(c) or u.dtype != velocity[0].dtype or u.device != velocity[0].device:
                raise ValueError('channel velocity shape/device/dtype mismatch')
