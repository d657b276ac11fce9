"""Shared pytest configuration: the ``gpu`` marker and fixture loading."""
import sys
from pathlib import Path
import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / 'tests' / 'golden'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


def golden(name):
    with np.load(GOLDEN / f'{name}.npz') as z:
        return {k: z[k] for k in z.files}


@pytest.fixture
def load_golden():
    return golden
