"""In-tree build of libgrappolo_b200.so for sm_100a (nvcc cross-compiles; no GPU needed)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libgrappolo_b200.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')

SOURCES = ['engine.cu', 'compat.cpp']
HEADERS = ['glv_common.cuh', 'sweep.cuh', 'phase_kernels.cuh', 'persist.cuh', 'recolor.cuh',
           'batch.cuh', 'batch_kernels.cuh', 'gate.cuh', 'csr_build.cuh', 'compare.cuh',
           'coarsen_hash.cuh']
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '--fmad=false',
         '-std=c++17', '-Xcompiler', '-fPIC', '-cudart', 'static',
         f'-I{os.path.join(ROOT, "include")}', f'-I{CSRC}']


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(ROOT, 'include', f) for f in os.listdir(os.path.join(ROOT, 'include'))]
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + '.o')
        cmd = [NVCC, *FLAGS, '-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = OUT + '.tmp'
    cmd = [NVCC, *FLAGS, '-shared', *objs, '-o', tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    for o in objs:
        os.remove(o)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
