"""B200-native (sm_100a) IB-transfer and MAC-multigrid hot path of AFSI_GPU.

Host code is Python/PyTorch mirroring the ``afsi_torch`` interfaces; every
compute step runs in the hand-written CUDA library ``libafsi_b200.so`` reached
through the C-ABI of ``include/afsi_b200.h``.

Modules
-------
cuda_ib            drop-in for ``afsi_torch.mac.cuda_ib`` (+ binning kernels)
p2_cuda_transfer   drop-in for ``afsi_torch.mac.p2_cuda_transfer`` (+ P2Transfer, FP32
                   and deterministic modes)
p1_csr             P1 hash contraction to CSR, cached-pattern maintenance, P1CSRTransfer
multigrid          GeometricMultigrid / ChannelMultigrid / DirichletMultigrid / RefinedMultigrid /
                   B200Kernels / MGOptions (Jacobi or red-black smoothing)
mass               consistent-mass Jacobi-PCG (MassSolver / GraphMassSolver)
helmholtz          CN Helmholtz kernels and workspace, Stokes residual reductions
batch              batching form: many 2D instances per step, autotuned schedule
serving            serving form: continuous-batching request loop
grid               MACGrid / ChannelGrid
quadrature         adaptive conical P2 / P1 interaction rules
synthetic          seeded inputs of the benchmark configurations
dropin             switch an installed ``afsi_torch`` onto these kernels
"""
from .grid import MACGrid, ChannelGrid
from .multigrid import MGOptions, GeometricMultigrid, ChannelMultigrid, B200Kernels

__all__ = ['MACGrid', 'ChannelGrid', 'MGOptions', 'GeometricMultigrid', 'ChannelMultigrid', 'B200Kernels']
