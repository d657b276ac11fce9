"""B200-native (sm_100a) IB-transfer and MAC-multigrid hot path of AFSI_GPU.

Host code is Python/PyTorch mirroring the ``afsi_torch`` interfaces; every
compute step runs in the hand-written CUDA library ``libafsi_b200.so`` reached
through the C-ABI of ``include/afsi_b200.h``.

Modules
-------
cuda_ib            drop-in for ``afsi_torch.mac.cuda_ib`` (+ binning kernels)
p2_cuda_transfer   drop-in for ``afsi_torch.mac.p2_cuda_transfer`` (+ P2Transfer)
multigrid          GeometricMultigrid / ChannelMultigrid / B200Kernels / MGOptions
grid               MACGrid / ChannelGrid
quadrature         adaptive conical P2 interaction rules
synthetic          seeded inputs of the benchmark configurations
dropin             switch an installed ``afsi_torch`` onto these kernels
"""
from .grid import MACGrid, ChannelGrid
from .multigrid import MGOptions, GeometricMultigrid, ChannelMultigrid, B200Kernels

__all__ = ['MACGrid', 'ChannelGrid', 'MGOptions', 'GeometricMultigrid', 'ChannelMultigrid', 'B200Kernels']
