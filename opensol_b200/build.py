"""Build libopensol_fdtd.so in-tree with nvcc for sm_100a (``python -m opensol_b200.build``).

The library is written next to the package (opensol_b200/_lib/) so it travels with the source tree; nothing is
installed into site-packages.  Each CUDA source is compiled to its own object (opensol_b200/_lib/obj/, in parallel,
and again only when the source or a header it includes changed), then the objects are linked.  Field kernels are
compiled with -fmad=false: every multiply and add is rounded on its own, in the order open_sol's CPU backend
evaluates it.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB_DIR = os.path.join(HERE, '_lib')
OBJ_DIR = os.path.join(LIB_DIR, 'obj')
LIB_NAME = 'libopensol_fdtd.so'
SOURCES = ['common.cu', 'fdtd2d.cu', 'fdtd3d.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-fmad=false', '-Xcompiler', '-fPIC', '-Xcompiler', '-O2']
_INCLUDE = re.compile(r'^\s*#include\s+"([^"]+)"', re.M)


def nvcc_path() -> str:
    for candidate in (shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError('nvcc not found: the CUDA toolkit is required to build libopensol_fdtd.so')


def sources():
    return [os.path.join(CSRC, name) for name in SOURCES]


def dependencies(path, seen=None):
    """The file and every file it includes with #include "...", recursively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        text = f.read()
    for name in _INCLUDE.findall(text):
        dependencies(os.path.join(os.path.dirname(path), name), seen)
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    built = os.path.getmtime(target)
    return any(os.path.getmtime(d) > built for d in deps)


def needs_build(target: str) -> bool:
    deps = set()
    for src in sources():
        deps |= dependencies(src)
    return _stale(target, deps)


def build(force: bool = False, verbose: bool = True, extra_flags=None) -> str:
    """Compile every CUDA source into one shared library; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    target = os.path.join(LIB_DIR, LIB_NAME)
    nvcc = nvcc_path()
    flags = list(extra_flags or []) + FLAGS
    jobs, objects = [], []
    for src in sources():
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + '.o')
        objects.append(obj)
        if force or _stale(obj, dependencies(src)):
            cmd = [nvcc, *ARCH, *flags, '-c', '-o', obj + '.tmp', src]
            if verbose:
                print(' '.join(cmd), flush=True)
            jobs.append((subprocess.Popen(cmd, cwd=CSRC), obj))
    failed = [obj for proc, obj in jobs if proc.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f'nvcc ({", ".join(os.path.basename(o) for o in failed)})')
    for _, obj in jobs:
        os.replace(obj + '.tmp', obj)
    if jobs or force or _stale(target, objects):
        cmd = [nvcc, *ARCH, '-shared', '-o', target + '.tmp', *objects, '-lcudart']
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.run(cmd, check=True, cwd=CSRC)
        os.replace(target + '.tmp', target)
    return target


if __name__ == '__main__':
    build(force='--force' in sys.argv)
