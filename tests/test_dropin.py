"""The drop-in switch rebinds afsi-torch's call targets (CPU; needs the reference source)."""
import os
import sys
import pytest

# the reference's src directory; the tests skip when it is not given
REF = os.environ.get('AFSI_TORCH_SRC', '')


@pytest.fixture
def afsi_torch():
    if not REF or not os.path.isdir(os.path.join(REF, 'afsi_torch')):
        pytest.skip('afsi-torch source not available (set AFSI_TORCH_SRC)')
    sys.path.insert(0, REF)
    try:
        import afsi_torch.mac.cuda_ib  # noqa: F401
        yield
    finally:
        sys.path.remove(REF)


def test_install_rebinds_ib_operators_and_mg_kernels(afsi_torch):
    import afsi_torch.mac.cuda_ib as ref_ib
    import afsi_torch.mac.p2_cuda_transfer as ref_p2
    from afsi_gpu_b200 import dropin, cuda_ib, p2_cuda_transfer
    from afsi_gpu_b200.multigrid import B200Kernels
    original = ref_ib.compact_gather
    dropin.install()
    try:
        assert ref_ib.compact_gather is cuda_ib.compact_gather
        assert ref_ib.indexed_spread is cuda_ib.indexed_spread
        assert ref_p2.assemble_velocity is p2_cuda_transfer.assemble_velocity
        from afsi_torch.mac._triton_mg import TritonKernels
        k = TritonKernels()
        assert isinstance(k, B200Kernels) and k.dim == 3
        from afsi_torch.mac2d._triton_mg import TritonKernels as Channel
        assert Channel().dim == 2
        import afsi_torch.mac.compact_transfer as ref_compact
        import afsi_torch.mac.mass_graph as ref_graph
        import afsi_torch.mac2d.transfer as ref_2d
        from afsi_gpu_b200 import mass
        assert ref_compact.MassSolver is mass.MassSolver and ref_graph.GraphMassSolver is mass.GraphMassSolver
        assert ref_2d.MassSolver is mass.MassSolver and ref_2d.GraphMassSolver is mass.GraphMassSolver
        from afsi_gpu_b200 import helmholtz
        from afsi_torch.mac._triton_helmholtz import HelmholtzKernels as HK
        from afsi_torch.mac._triton_stokes import residual_partial as rp
        assert HK is helmholtz.HelmholtzKernels and rp is helmholtz.residual_partial
        import afsi_torch.mac.cached_transfer_assembly as ref_cached
        from afsi_gpu_b200 import p1_csr
        assert ref_cached.finish_cached_component is p1_csr.finish_cached_component
        assert p1_csr.PatternBudgetExceeded is ref_cached.PatternBudgetExceeded
    finally:
        dropin.uninstall()
    assert ref_ib.compact_gather is original
    import afsi_torch.mac.mass_solver as ref_mass
    assert ref_compact.MassSolver is ref_mass.MassSolver and ref_2d.MassSolver is ref_mass.MassSolver
