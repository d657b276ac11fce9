"""Compile the sm_100a C-ABI library ``libafsi_b200.so`` in-tree with nvcc.

The library has no PyTorch dependency: plain CUDA C++ behind the ``extern "C"``
entry points declared in ``include/afsi_b200.h``.
"""
import os
import shutil
import subprocess
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / 'csrc'
LIBRARY = PACKAGE / 'libafsi_b200.so'
SOURCES = ('api.cu', 'prepare.cu', 'transfer.cu', 'p2.cu', 'mg.cu', 'mg_persistent.cu', 'csr.cu', 'mass.cu', 'batch.cu', 'stokes.cu', 'det_spread.cu', 'batch_refine.cu', 'fgmres.cu', 'fe_fused.cu')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '--fmad=false', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-O3',
         '--expt-relaxed-constexpr']


def nvcc():
    cuda = os.environ.get('CUDA_HOME', '/usr/local/cuda')
    path = Path(cuda) / 'bin' / 'nvcc'
    return str(path) if path.exists() else shutil.which('nvcc') or 'nvcc'


def sources():
    return [CSRC / s for s in SOURCES]


def stale():
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    deps = list(sources()) + list(CSRC.glob('*.cuh')) + [ROOT / 'include' / 'afsi_b200.h']
    return any(d.stat().st_mtime > built for d in deps)


def build(*, force=False, verbose=False, ptxas_info=False):
    """Compile every source and link ``libafsi_b200.so`` (no-op when fresh)."""
    if not force and not stale():
        return LIBRARY
    objdir = PACKAGE / '_build'
    objdir.mkdir(exist_ok=True)
    objects = []
    for src in sources():
        obj = objdir / (src.stem + '.o')
        cmd = [nvcc(), *ARCH, *FLAGS, '-I', str(ROOT / 'include'), '-c', str(src), '-o', str(obj)]
        if ptxas_info:
            cmd.insert(1, '-Xptxas=-v')
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = LIBRARY.with_suffix('.so.tmp')
    cmd = [nvcc(), *ARCH, '-shared', '-o', str(tmp), *objects, '-lcudart']
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == '__main__':
    import sys
    build(force=True, verbose=True, ptxas_info='-v' in sys.argv)
    print(LIBRARY)
