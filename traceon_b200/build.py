"""Builds libtraceon_b200.so (all CUDA sources in csrc/) for sm_100a in-tree.

    python -m traceon_b200.build

nvcc cross-compiles without a GPU.  The CUDA runtime is linked statically
(nvcc's default), so the library does not depend on which libcudart the host
process (e.g. PyTorch) loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libtraceon_b200.so')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')

SOURCES = ['tb_bem.cu', 'tb_lu.cu', 'tb_trace.cu', 'tb_compat.cu', 'tb_mlp.cu', 'tb_lu_mixed.cu', 'tb_post.cu', 'tb_batch.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-shared', '--expt-relaxed-constexpr',
         '-Xptxas', '-v']


def nvcc() -> str:
    for c in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return 'nvcc'


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, 'traceon_b200.h')]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, *FLAGS, '-I', INCLUDE, '-o', LIB + '.tmp',
           *[os.path.join(CSRC, s) for s in SOURCES]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError('nvcc failed building libtraceon_b200.so')
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)
    print(LIB)
