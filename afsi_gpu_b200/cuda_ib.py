"""Drop-in counterparts of ``afsi_torch.mac.cuda_ib`` on the B200 kernels.

Same function names, argument meaning, output ownership and error behaviour as
``afsi_torch/mac/cuda_ib.py:38-112`` and the ``afsi_ib_cuda`` operator schemas
(``mac/csrc/transfer.cpp:48-57``): outputs of the gathers/spreads are freshly
allocated, tensors are made contiguous, kernels run on PyTorch's current CUDA
stream, and a CPU tensor is rejected (no silent CPU fallback,
``mac/cuda_ib.py:63-66``).  Stencil indices that leave the grid do not trap
the device (the reference uses ``CUDA_KERNEL_ASSERT``); the kernels set a bit in
the device status word, which :func:`check` turns into a ``RuntimeError``.

Beyond the reference operators this module exposes the binning kernels
(:func:`compact_prepare`, :func:`prepare2d`), which the reference runs as torch
expressions.
"""
from dataclasses import dataclass
import torch
from . import _lib
from ._lib import call, ptr, stream, dtype_code


def build(*, verbose=False):
    """Compile (if needed) and load the native library; call before graph capture."""
    if torch.cuda.is_available() and torch.cuda.is_current_stream_capturing():
        raise RuntimeError('build the B200 IB library before CUDA Graph capture')
    from .build import build as _build
    _build(verbose=verbose)
    _lib.load()


def require_cuda(tensor):
    _lib.require_cuda(tensor)


def check(device=None, *, clear=True):
    """Raise if a kernel flagged an out-of-range stencil or support violation.

    Synchronises with the device (reads the status word)."""
    word = _lib.status_word(device if device is not None else torch.cuda.current_device())
    value = int(word.item())
    if clear:
        word.zero_()
    if value & _lib.FLAG_INDEX:
        raise RuntimeError('IB stencil index outside the MAC grid or node range')
    if value & _lib.FLAG_SUPPORT:
        raise ValueError('MAC IB support reaches a wall or is nonfinite; enlarge/refine the fluid box')
    return value


def _field(t):
    if t.dtype not in (torch.float32, torch.float64):
        raise RuntimeError('IB supports float32/float64')
    return t


def _same(t, like, dtype):
    if not t.is_cuda or t.device != like.device:
        raise RuntimeError('IB transfer requires one CUDA device')
    if t.dtype != dtype:
        raise RuntimeError('IB transfer requires contiguous matching tensors')
    if t.requires_grad:
        raise RuntimeError('IB forward transfer does not register autograd')
    return t.contiguous()


# ------------------------------------------------------------- raw operators
# Schemas of afsi_ib_cuda.{indexed_gather, indexed_spread, compact_gather,
# compact_spread} (mac/csrc/transfer.cpp:48-57) and their checks (:9-41).

def op_indexed_gather(field, indices, weights):
    field = _same(_field(field), field, field.dtype)
    indices, weights = _same(indices, field, torch.int64), _same(weights, field, field.dtype)
    if field.dim() != 2 or field.shape[1] == 0:
        raise RuntimeError('IB indexed field must be N x C')
    if indices.dim() != 2 or indices.shape[1] == 0 or indices.shape != weights.shape:
        raise RuntimeError('IB indexed stencil shape mismatch')
    if field.shape[0] == 0:
        raise RuntimeError('empty IB grid')
    P, K = indices.shape
    out = torch.empty((P, field.shape[1]), device=field.device, dtype=field.dtype)
    call('afsi_b200_indexed_gather', ptr(field), field.shape[0], field.shape[1], ptr(indices), ptr(weights),
         P, K, ptr(out), ptr(_lib.status_word(field.device)), dtype_code(field.dtype), stream(field.device))
    return out


def op_indexed_spread(field, indices, weights, size, volume):
    field = _same(_field(field), field, field.dtype)
    indices, weights = _same(indices, field, torch.int64), _same(weights, field, field.dtype)
    if field.dim() != 2 or field.shape[1] == 0:
        raise RuntimeError('IB indexed field must be N x C')
    if indices.dim() != 2 or indices.shape[1] == 0 or indices.shape != weights.shape:
        raise RuntimeError('IB indexed stencil shape mismatch')
    if not (size > 0 and volume > 0 and volume == volume and volume != float('inf')):
        raise RuntimeError('invalid IB output size/volume')
    if field.shape[0] != indices.shape[0]:
        raise RuntimeError('IB spread point count mismatch')
    out = torch.zeros((size, field.shape[1]), device=field.device, dtype=field.dtype)
    call('afsi_b200_indexed_spread', ptr(field), field.shape[0], field.shape[1], ptr(indices), ptr(weights),
         indices.shape[1], size, float(volume), ptr(out), ptr(_lib.status_word(field.device)),
         dtype_code(field.dtype), stream(field.device))
    return out


def _compact_checks(field, base, phi, nx, ny, nz, volume, spread):
    field = _same(_field(field), field, field.dtype)
    base, phi = _same(base, field, torch.int64), _same(phi, field, field.dtype)
    if field.dim() != 1 or base.dim() != 2 or base.shape[1] != 3:
        raise RuntimeError('invalid compact IB field/base')
    if phi.dim() != 3 or phi.shape[0] != base.shape[0] or phi.shape[1] != 3 or phi.shape[2] != 4:
        raise RuntimeError('invalid compact IB weights')
    if not (nx > 0 and ny > 0 and nz > 0 and volume > 0):
        raise RuntimeError('invalid compact grid/volume')
    if field.numel() != (base.shape[0] if spread else nx * ny * nz):
        raise RuntimeError('compact IB field length mismatch')
    return field, base, phi


def op_compact_gather(field, base, phi, nx, ny, nz):
    field, base, phi = _compact_checks(field, base, phi, nx, ny, nz, 1., False)
    out = torch.empty(base.shape[0], device=field.device, dtype=field.dtype)
    call('afsi_b200_compact_gather', ptr(field), ptr(base), ptr(phi), base.shape[0], nx, ny, nz, ptr(out),
         ptr(_lib.status_word(field.device)), dtype_code(field.dtype), stream(field.device))
    return out


def op_compact_spread(field, base, phi, nx, ny, nz, volume):
    field, base, phi = _compact_checks(field, base, phi, nx, ny, nz, volume, True)
    out = torch.zeros(nx * ny * nz, device=field.device, dtype=field.dtype)
    call('afsi_b200_compact_spread', ptr(field), ptr(base), ptr(phi), base.shape[0], nx, ny, nz, float(volume),
         ptr(out), ptr(_lib.status_word(field.device)), dtype_code(field.dtype), stream(field.device))
    return out


# ----------------------------------------------------- Python-level wrappers
# afsi_torch/mac/cuda_ib.py:69-90

def indexed_gather(field, indices, weights):
    require_cuda(field)
    return op_indexed_gather(field.contiguous(), indices.contiguous(), weights.contiguous())


def indexed_spread(field, indices, weights, size, volume=1.):
    require_cuda(field)
    return op_indexed_spread(field.contiguous(), indices.contiguous(), weights.contiguous(), size, float(volume))


def compact_gather(grid, velocity, stencil):
    require_cuda(velocity[0])
    return torch.stack([op_compact_gather(u.contiguous().view(-1), stencil.base[c].contiguous(),
                                          stencil.phi[c].contiguous(), *grid.face_shape(c))
                        for c, u in enumerate(velocity)], -1)


def compact_spread(grid, force, stencil):
    require_cuda(force)
    return tuple(op_compact_spread(force[:, c].contiguous(), stencil.base[c].contiguous(),
                                   stencil.phi[c].contiguous(), *grid.face_shape(c),
                                   float(grid.volume)).view(grid.face_shape(c)) for c in range(3))


# ------------------------------------------------------------------ binning

@dataclass(frozen=True)
class CompactStencil:
    """base (L,P,3) int64 and phi (L,P,3,4); L=3 component tables
    (``mac/compact_transfer.py:11-18``) or L=2 shared face/centre tables
    (``mac/shared_stencil.py:8-19``)."""
    base: torch.Tensor
    phi: torch.Tensor
    layout: str = 'component'

    @property
    def storage_bytes(self):
        return self.base.numel() * self.base.element_size() + self.phi.numel() * self.phi.element_size()

    def expanded(self):
        if self.layout != 'shared':
            return self
        base = torch.stack([torch.stack([self.base[int(a != c), :, a] for a in range(3)], -1) for c in range(3)])
        phi = torch.stack([torch.stack([self.phi[int(a != c), :, a, :] for a in range(3)], 1) for c in range(3)])
        return CompactStencil(base, phi, 'component')


def compact_prepare(grid, points, *, layout='component', phi_form='clamped', check_support=True):
    """Binning + weights of ``mac/compact_transfer.py:21-26`` (``from_points``),
    with the support screen of ``compact_transfer.py:94-96`` fused.

    ``phi_form='clamped'`` is the torch kernel (``ib.py:57-67``); ``'radical'``
    the shared radical of the reference CUDA/Triton prepares.  Raises
    ``ValueError`` (after a device sync) when a point's support leaves the grid.
    """
    require_cuda(points)
    points = points.contiguous()
    if points.dim() != 2 or points.shape[1] != 3:
        raise ValueError('points must be (P,3)')
    P = points.shape[0]
    if layout == 'component':
        origins = [grid.face_origin(c) for c in range(3)]
    elif layout == 'shared':
        origins = [grid.origin, tuple(o + .5 * h for o, h in zip(grid.origin, grid.spacing))]
    else:
        raise ValueError('layout must be component or shared')
    L = len(origins)
    base = torch.empty((L, P, 3), device=points.device, dtype=torch.int64)
    phi = torch.empty((L, P, 3, 4), device=points.device, dtype=points.dtype)
    word = _lib.status_word(points.device)
    if check_support:
        word.zero_()
    call('afsi_b200_compact_prepare', ptr(points), P, L, _lib.doubles(sum(map(list, origins), [])),
         _lib.doubles(grid.spacing), _lib.doubles(grid.origin), _lib.int64s(grid.shape),
         _lib.PHI_RADICAL if phi_form == 'radical' else _lib.PHI_CLAMPED, ptr(base), ptr(phi), ptr(word),
         dtype_code(points.dtype), stream(points.device))
    if check_support and P and int(word.item()) & _lib.FLAG_SUPPORT:
        word.zero_()
        raise ValueError('MAC IB support reaches a wall or is nonfinite; enlarge/refine the fluid box')
    return CompactStencil(base, phi, layout)


@dataclass(frozen=True)
class Stencil2D:
    """Reflected 2D stencils (``mac2d/transfer.py:12-15``): per component ids
    (P,16) int64 and signed weights (P,16)."""
    indices: tuple
    weights: tuple


def prepare2d(grid, points, *, check_support=True):
    """``TriangleTransfer._prepare`` (``mac2d/transfer.py:61-81``) with the
    support screen of ``mac2d/transfer.py:97-101`` fused."""
    require_cuda(points)
    points = points.contiguous()
    if points.dim() != 2 or points.shape[1] != 2:
        raise ValueError('points must be (P,2)')
    P = points.shape[0]
    ids = torch.empty((2, P, 16), device=points.device, dtype=torch.int64)
    w = torch.empty((2, P, 16), device=points.device, dtype=points.dtype)
    word = _lib.status_word(points.device)
    if check_support:
        word.zero_()
    hx, hy = grid.spacing
    call('afsi_b200_indexed_prepare2d', ptr(points), P, grid.shape[0], grid.shape[1], hx, hy,
         grid.lengths[0], grid.lengths[1], ptr(ids), ptr(w), ptr(word), dtype_code(points.dtype),
         stream(points.device))
    if check_support and P and int(word.item()) & _lib.FLAG_SUPPORT:
        word.zero_()
        raise ValueError('valve IB points leave the channel support region')
    return Stencil2D((ids[0], ids[1]), (w[0], w[1]))


def spread2d(grid, force, stencil):
    """``TriangleTransfer._spread`` CUDA branch (``mac2d/transfer.py:108-112``):
    point forces (P,2) -> (u, v) face fields divided by the cell area."""
    return tuple(indexed_spread(force[:, c:c + 1], stencil.indices[c], stencil.weights[c],
                                grid.face_shape(c)[0] * grid.face_shape(c)[1], grid.volume)
                 .reshape(grid.face_shape(c)) for c in range(2))


def gather2d(velocity, stencil):
    """``TriangleTransfer._gather`` CUDA branch (``mac2d/transfer.py:122-124``)."""
    return torch.cat([indexed_gather(u.reshape(-1, 1), ids, w)
                      for u, ids, w in zip(velocity, stencil.indices, stencil.weights)], -1)


def contract(stencil, group, component, offset, low, width, prefix, count, face_shape, workspace, cache=None):
    """``mac/cuda_ib.py:93-106``: P1 box-site contraction into the hash table."""
    from .p1_csr import contract as _contract
    _contract(stencil, group, component, offset, low, width, prefix, count, face_shape, workspace, cache)


def hash_accumulate(keys, values, workspace):
    """``mac/cuda_ib.py:109-112``: insert a (key, value) stream into the table."""
    from .p1_csr import hash_accumulate as _accumulate
    _accumulate(keys, values, workspace)
