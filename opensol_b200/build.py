"""Build libopensol_fdtd.so in-tree with nvcc for sm_100a (``python -m opensol_b200.build``).

The library is written next to the package (opensol_b200/_lib/) so it travels with the source tree; nothing is
installed into site-packages.  Field kernels are compiled with -fmad=false: every multiply and add is rounded on its
own, in the order open_sol's CPU backend evaluates it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB_DIR = os.path.join(HERE, '_lib')
LIB_NAME = 'libopensol_fdtd.so'
SOURCES = ['common.cu', 'fdtd2d.cu', 'fdtd3d.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_path() -> str:
    for candidate in (shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError('nvcc not found: the CUDA toolkit is required to build libopensol_fdtd.so')


def sources():
    return [os.path.join(CSRC, name) for name in SOURCES]


def needs_build(target: str) -> bool:
    if not os.path.exists(target):
        return True
    built = os.path.getmtime(target)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, 'include', 'opensol_fdtd.h')]
    return any(os.path.getmtime(d) > built for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = True, extra_flags=None) -> str:
    """Compile every CUDA source into one shared library; returns its path."""
    os.makedirs(LIB_DIR, exist_ok=True)
    target = os.path.join(LIB_DIR, LIB_NAME)
    if not force and not needs_build(target):
        return target
    cmd = [nvcc_path(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-fmad=false', '-Xcompiler', '-fPIC',
           '-Xcompiler', '-O2', '-shared', '-o', target + '.tmp', *sources(), '-lcudart']
    if extra_flags:
        cmd[1:1] = list(extra_flags)
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(target + '.tmp', target)
    return target


if __name__ == '__main__':
    build(force='--force' in sys.argv)
