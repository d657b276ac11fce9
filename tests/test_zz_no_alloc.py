"""The no-allocation residual norm agrees with the scratch-using one (B200).

``afsi_b200_mg_residual_norm_noalloc`` exists for callers that cannot allocate
device memory when they need a residual norm: host applications that hand the
library only their own preallocated buffers, embeddings without a caching
allocator, or code that cannot afford the device synchronisation of a
cudaMalloc.  It keeps its
reduction scratch in a fixed device array inside the library instead of in
caller-provided memory.  This file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes
import numpy as np
import pytest
import torch
from afsi_gpu_b200 import _lib, synthetic
from afsi_gpu_b200.grid import MACGrid, ChannelGrid
from afsi_gpu_b200.multigrid import GeometricMultigrid, ChannelMultigrid

pytestmark = pytest.mark.gpu


def _noalloc_norm(p, rhs, spacing, bc):
    dim = p.dim()
    out = torch.full((1,), float('nan'), device=p.device, dtype=torch.float64)
    shape = list(p.shape) + [1] * (3 - dim)
    h2 = [h * h for h in spacing] + [1.] * (3 - dim)
    _lib.call('afsi_b200_mg_residual_norm_noalloc', p.data_ptr(), rhs.data_ptr(), _lib.int64s(shape),
              _lib.doubles(h2), dim, bc, out.data_ptr(), _lib.dtype_code(p.dtype), _lib.stream(p.device))
    return out[0]


def _scratch_norm(solver, p, rhs):
    solver.initialize(p, rhs)
    return solver.residual_norm().clone()


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_noalloc_residual_norm_matches_scratch_version_twice_in_a_row(dtype):
    grid = MACGrid((64, 48, 32), (1., .75, .5))
    mg = GeometricMultigrid(grid, dtype=dtype, backend='b200')
    rng = np.random.default_rng(21)
    for trial in range(2):  # the shared array keeps the last call's contents
        p = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda', dtype=dtype)
        rhs = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda', dtype=dtype)
        got = _noalloc_norm(p, rhs, grid.spacing, _lib.BC_NEUMANN)
        ref = _scratch_norm(mg, p, rhs)
        # same kernel, same launch geometry, same partial order: bitwise equal
        assert got.item() == ref.item() > 0


def test_noalloc_residual_norm_2d_channel_and_rejects_large_grids():
    grid = ChannelGrid((256, 64), (8., 1.61))
    mg = ChannelMultigrid(grid, backend='b200')
    rng = np.random.default_rng(22)
    for trial in range(2):
        p = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda')
        rhs = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda')
        got = _noalloc_norm(p, rhs, grid.spacing, _lib.BC_CHANNEL)
        assert got.item() == _scratch_norm(mg, p, rhs).item()
    big = torch.zeros((2048, 4096), device='cuda')  # 2^23 cells: 32768 reduction blocks
    with pytest.raises(RuntimeError, match='at most 4096'):
        _noalloc_norm(big, big, (1 / 2048, 1 / 4096), _lib.BC_CHANNEL)


@pytest.mark.parametrize('case', ['dirichlet', 'periodic'])
def test_noalloc_residual_norm_other_boundaries(case):
    """Dirichlet (3D) and periodic-x (2D) against the scratch-using norm of
    their own solvers, bitwise."""
    from afsi_gpu_b200.multigrid import DirichletMultigrid
    rng = np.random.default_rng(23)
    if case == 'dirichlet':
        grid = MACGrid((32, 32, 32), (1., 1., 1.))
        mg, bc = DirichletMultigrid(grid, backend='b200'), _lib.BC_DIRICHLET
    else:
        grid = ChannelGrid((128, 32), (4., 1.), periodic=True)
        mg, bc = ChannelMultigrid(grid, backend='b200'), _lib.BC_PERIODIC
    for trial in range(2):
        p = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda')
        rhs = torch.as_tensor(rng.standard_normal(grid.shape), device='cuda')
        got = _noalloc_norm(p, rhs, grid.spacing, bc)
        assert got.item() == _scratch_norm(mg, p, rhs).item() > 0


def test_noalloc_residual_norm_rejects_large_3d_sections():
    """A 3D grid whose y-z section needs more than 4096 reduction blocks."""
    big = torch.zeros((2, 1024, 1040), device='cuda')
    with pytest.raises(RuntimeError, match='at most 4096'):
        _noalloc_norm(big, big, (.5, 1 / 1024, 1 / 1040), _lib.BC_NEUMANN)
