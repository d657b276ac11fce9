"""Switch an installed afsi-torch onto the B200 kernels.

``install()`` rebinds, in place, the functions the reference resolves at call
time:

* ``afsi_torch.mac.cuda_ib.{build, require_cuda, indexed_gather,
  indexed_spread, compact_gather, compact_spread, contract,
  hash_accumulate}`` (``mac/cuda_ib.py:38-112``), which the P1 hash assembly
  (``mac/hash_transfer_assembly.py:84-99``) imports at call time;
* ``afsi_torch.mac.p2_cuda_transfer.{prepare, spread, assemble_velocity}``
  (``mac/p2_cuda_transfer.py:18-60``), which ``AdaptiveFETransfer`` imports
  inside its methods;
* the CUDA kernel objects of the multigrid workspaces: ``MGWorkspace`` and
  ``ChannelWorkspace`` import ``TritonKernels`` from ``mac._triton_mg`` /
  ``mac2d._triton_mg`` when they are built (``mac/mg_workspace.py:36-47``,
  ``mac2d/mg_workspace.py:28-40``); those modules are replaced by shims whose
  ``TritonKernels`` is the B200 kernel object;
* the CN Helmholtz kernel object and the Stokes reductions, which
  ``HelmholtzWorkspace`` and ``StokesWorkspace`` import when they are built or
  measure (``mac/helmholtz.py:44-47``, ``mac/stokes_workspace.py:50,86,97``):
  ``mac._triton_helmholtz`` and ``mac._triton_stokes`` are replaced by shims
  holding the B200 ``HelmholtzKernels`` and partial functions;
* the cached CSR pattern maintenance, ``finish_cached_component`` and
  ``numeric_snapshot`` of ``mac.cached_transfer_assembly`` (called through
  that module's globals by ``assemble_component_cached``, :186-280), with the
  reference's ``PatternBudgetExceeded`` raised so that its handler applies;
* the consistent-mass solvers: ``MassSolver`` as bound in
  ``mac.compact_transfer`` and ``mac2d.transfer`` (imported there at module
  load, ``mac/compact_transfer.py:7``, ``mac2d/transfer.py:10-11``),
  ``GraphMassSolver`` in ``mac.mass_graph`` (imported at call time,
  ``mac/compact_transfer.py:89``) and in ``mac2d.transfer``.

Nothing is copied from the reference.  ``uninstall()`` restores the originals.
"""
import sys
import types

_saved = {}


def _shim(name, bc):
    from .multigrid import B200Kernels

    def factory():
        return B200Kernels(bc)

    module = types.ModuleType(name)
    module.TritonKernels = factory
    module.__doc__ = f'B200 kernel objects standing in for {name}'
    return module


def install():
    """Point afsi_torch's CUDA IB operators and MG kernel objects at this library."""
    import afsi_torch.mac.cuda_ib as ref_ib
    import afsi_torch.mac.p2_cuda_transfer as ref_p2
    from . import cuda_ib, p2_cuda_transfer
    for name in ('build', 'require_cuda', 'indexed_gather', 'indexed_spread', 'compact_gather', 'compact_spread',
                 'contract', 'hash_accumulate'):
        _saved.setdefault(('cuda_ib', name), getattr(ref_ib, name))
        setattr(ref_ib, name, getattr(cuda_ib, name))
    for name in ('prepare', 'spread', 'assemble_velocity'):
        _saved.setdefault(('p2', name), getattr(ref_p2, name))
        setattr(ref_p2, name, getattr(p2_cuda_transfer, name))
    import importlib
    from . import mass
    for module, name in (('afsi_torch.mac.compact_transfer', 'MassSolver'),
                         ('afsi_torch.mac.mass_graph', 'GraphMassSolver'),
                         ('afsi_torch.mac2d.transfer', 'MassSolver'),
                         ('afsi_torch.mac2d.transfer', 'GraphMassSolver')):
        target = importlib.import_module(module)
        _saved.setdefault(('attr', module, name), getattr(target, name))
        setattr(target, name, getattr(mass, name))
    from . import helmholtz, p1_csr
    import afsi_torch.mac.cached_transfer_assembly as ref_cached
    for name in ('finish_cached_component', 'numeric_snapshot'):
        _saved.setdefault(('attr', 'afsi_torch.mac.cached_transfer_assembly', name), getattr(ref_cached, name))
        setattr(ref_cached, name, getattr(p1_csr, name))
    # the reference's assembly catches its own budget exception class
    _saved.setdefault(('attr', 'afsi_gpu_b200.p1_csr', 'PatternBudgetExceeded'), p1_csr.PatternBudgetExceeded)
    p1_csr.PatternBudgetExceeded = ref_cached.PatternBudgetExceeded
    for module, names in (('afsi_torch.mac._triton_helmholtz', ('HelmholtzKernels',)),
                          ('afsi_torch.mac._triton_stokes', ('start_partial', 'residual_partial',
                                                            'pressure_input_partial', 'pressure_norm_partial'))):
        _saved.setdefault(('module', module), sys.modules.get(module))
        shim = types.ModuleType(module)
        shim.__doc__ = f'B200 kernels standing in for {module}'
        for name in names:
            setattr(shim, name, getattr(helmholtz, name))
        sys.modules[module] = shim
        parent, _, leaf = module.rpartition('.')
        if parent in sys.modules:
            setattr(sys.modules[parent], leaf, shim)
    for module, bc in (('afsi_torch.mac._triton_mg', 'neumann'), ('afsi_torch.mac2d._triton_mg', 'channel')):
        _saved.setdefault(('module', module), sys.modules.get(module))
        sys.modules[module] = _shim(module, bc)
        parent, _, leaf = module.rpartition('.')
        if parent in sys.modules:
            setattr(sys.modules[parent], leaf, sys.modules[module])


def uninstall():
    import afsi_torch.mac.cuda_ib as ref_ib
    import afsi_torch.mac.p2_cuda_transfer as ref_p2
    import importlib
    for key, value in list(_saved.items()):
        if key[0] == 'attr':
            setattr(importlib.import_module(key[1]), key[2], value)
            continue
        kind, name = key
        if kind == 'cuda_ib':
            setattr(ref_ib, name, value)
        elif kind == 'p2':
            setattr(ref_p2, name, value)
        else:
            if value is None:
                sys.modules.pop(name, None)
            else:
                sys.modules[name] = value
    _saved.clear()
