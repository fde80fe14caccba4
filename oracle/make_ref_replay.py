"""ORACLE -- BENCH / TEST INFRASTRUCTURE ONLY: the recipe of the reference-kernel replay's cubin.

Compiles open_sol's own 2D E_z RawKernels, update_h_kernel and update_e_kernel (the CUDA source strings
_UPDATE_H_SOURCE / _UPDATE_E_SOURCE of open_sol/physics/em/solvers/fdtd_ez_2d_kernels.py:23-122), unchanged, for
sm_100a into oracle/_ref/ez2d_rawkernels.cubin.  The strings are read from the reference tree where they lie (parsed
with ast, nothing imported or executed) and prefixed with the float32 preamble RealRawKernel adds
(open_sol/core/kernels.py:173-182); the combined source goes to a temporary file outside the repository, is compiled
with nvcc's defaults (contraction into FMA on, as NVRTC compiles a cupy RawKernel by default), and is deleted.  Only
the cubin is written under oracle/_ref/, which stays out of version control.

    python oracle/make_ref_replay.py /path/to/reference
"""
import ast
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, '_ref')
CUBIN = os.path.join(OUT_DIR, 'ez2d_rawkernels.cubin')
KERNEL_FILE = os.path.join('open_sol', 'physics', 'em', 'solvers', 'fdtd_ez_2d_kernels.py')
NAMES = ('_UPDATE_H_SOURCE', '_UPDATE_E_SOURCE')
PREAMBLE = 'typedef float real_t;\n#define REAL_IS_DOUBLE 0\n'


def kernel_sources(reference):
    """The reference's RawKernel source strings, in NAMES order."""
    path = os.path.join(reference, KERNEL_FILE)
    with open(path) as f:
        tree = ast.parse(f.read(), path)
    found = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name in NAMES and isinstance(node.value, ast.Constant) and isinstance(node.value.value, str):
                found[name] = node.value.value
    missing = [n for n in NAMES if n not in found]
    if missing:
        raise RuntimeError(f'{path}: no string constant {missing}')
    return [found[n] for n in NAMES]


def nvcc():
    for candidate in (shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError('nvcc not found')


def build(reference):
    os.makedirs(OUT_DIR, exist_ok=True)
    sources = kernel_sources(reference)
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, 'ez2d_rawkernels.cu')
        with open(src, 'w') as f:
            f.write(PREAMBLE + '\n'.join(sources))
        subprocess.run([nvcc(), '-cubin', '-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-o', CUBIN + '.tmp',
                        src], check=True)
    os.replace(CUBIN + '.tmp', CUBIN)
    return CUBIN


if __name__ == '__main__':
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_ref_replay.py /path/to/reference')
    print(build(reference))
