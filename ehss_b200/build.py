"""Build libehss_b200.so in-tree for B200 (sm_100a) with nvcc.

    python -m ehss_b200.build [--force] [--verbose]

The shared library lands next to this file so that it travels with the
source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
ROOT = HERE.parent
LIB = HERE / 'libehss_b200.so'
SOURCES = ['capi.cu', 'scene.cu', 'trace.cu', 'pa_grid.cu', 'compact.cu', 'noalloc.cu', 'sobol_host.cpp']
HEADERS = ['ehss_internal.cuh']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError('nvcc not found: the CUDA toolkit is required to build ehss_b200')


def stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / 'include' / 'ehss_b200.h', Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force=False, verbose=False, ptxas_verbose=False):
    if not force and not stale():
        return LIB
    tmp = LIB.with_suffix('.so.tmp')
    cmd = [nvcc(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '--shared', '-Xcompiler', '-fPIC',
           '-I', str(ROOT / 'include'), '-o', str(tmp), *[str(CSRC / s) for s in SOURCES], '-cudart', 'static']
    if ptxas_verbose:
        cmd[1:1] = ['-Xptxas', '-v']
    if verbose:
        print(' '.join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f'nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}')
    if verbose or ptxas_verbose:
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--ptxas', action='store_true', help='print register / spill / shared-memory use')
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))


if __name__ == '__main__':
    main()
