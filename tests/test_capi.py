"""The C-ABI library loads and exports every entry point the header declares (CPU)."""
import ctypes
import re
from pathlib import Path
import pytest
from afsi_gpu_b200 import _lib
from afsi_gpu_b200.build import build, LIBRARY

HEADER = Path(__file__).resolve().parents[1] / 'include' / 'afsi_b200.h'


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r'\b(afsi_b200_\w+)\s*\(', text)))


def test_library_builds_and_exports_every_declared_symbol():
    build()
    lib = ctypes.CDLL(str(LIBRARY))
    names = declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding covers exactly the declared entry points
    assert sorted(_lib.exported_symbols()) == names


def test_version_and_argument_errors_without_a_gpu():
    lib = _lib.load()
    assert lib.afsi_b200_version() >= 100
    # argument validation happens on the host before any launch
    with pytest.raises(RuntimeError, match='negative point count'):
        _lib.call('afsi_b200_compact_prepare', None, -1, 3, _lib.doubles([0] * 9), _lib.doubles([1] * 3),
                  _lib.doubles([0] * 3), _lib.int64s([8] * 3), 0, None, None, None, _lib.F64, None)
    with pytest.raises(RuntimeError, match='dtype'):
        _lib.call('afsi_b200_compact_gather', 1, 1, 1, 4, 8, 8, 8, 1, None, 7, None)
    with pytest.raises(RuntimeError, match='table bounds'):
        _lib.call('afsi_b200_p2_spread', 1, 10, 1, 5, 1, 4, 1, 1, 1, 10, 0, 1, 1, 1, 8, 8, 8, 1., None,
                  _lib.F64, None)
    plan = _lib.MGPlan()
    plan.dim, plan.bc, plan.levels = 3, _lib.BC_CHANNEL, 1
    with pytest.raises(RuntimeError, match='dim/boundary'):
        _lib.call('afsi_b200_mg_vcycles', ctypes.byref(plan), 1, None)
    # empty inputs are a no-op, not an error
    _lib.call('afsi_b200_indexed_gather', None, 4, 1, None, None, 0, 16, None, None, _lib.F64, None)


def test_cpu_tensors_are_rejected_not_computed():
    import torch
    from afsi_gpu_b200 import cuda_ib
    with pytest.raises(ValueError, match='CUDA'):
        cuda_ib.indexed_gather(torch.zeros(4, 1), torch.zeros(1, 16, dtype=torch.int64), torch.zeros(1, 16))
