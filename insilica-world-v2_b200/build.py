"""Build the isw CUDA library (libisw.so, in the package directory) for sm_100a with nvcc.

    python insilica-world-v2_b200/build.py [--verbose] [--check]

FP64 sources compile with -fmad=false (no fused multiply-add: every product rounds as the reference's --fmad=false
kernels do); host code with -ffp-contract=off for the same reason (the transport stencil's weights are computed on the
host). The mixed form's kernels (batch_mixed.cu) compile with fused multiply-adds. --check adds -DISW_CHECK (device-side bounds checks on gathered indices, for debugging).
"""
import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / 'csrc'
OUT = PKG / 'isw' / 'libisw.so'
BUILD = PKG / '_build'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
SOURCES = [  # (file, extra flags)
    ('grid.cu', ['-fmad=false']),
    ('layers.cu', ['-fmad=false']),
    ('transport.cu', ['-fmad=false']),
    ('dsum.cu', ['-fmad=false']),
    ('mesh.cu', ['-fmad=false', '-Xcompiler', '-fopenmp']),
    ('tiles.cu', ['-fmad=false']),
    ('batch.cu', ['-fmad=false']),
    ('batch_mixed.cu', ['-fmad=true']),     # the mixed form: fused multiply-adds allowed
]


def build(verbose=False, check=False, force=False):
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob('*.cuh')) + [PKG.parent / 'include' / 'isw.h']
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = []
    common = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-ffp-contract=off', '-Xptxas', '-v' if verbose else '-O3']
    if check:
        common += ['-DISW_CHECK']
    for src, extra in SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + '.o')
        objs.append(o)
        if not force and o.exists() and o.stat().st_mtime > max(s.stat().st_mtime, newest_header) and not check:
            continue
        cmd = [NVCC, '-c', str(s), '-o', str(o)] + common + extra
        if verbose:
            print(' '.join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    cmd = [NVCC, '-shared', '-o', str(OUT)] + [str(o) for o in objs] + ARCH + ['-cudart', 'static', '-lgomp']
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--check', action='store_true')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    try:
        print(build(a.verbose, a.check, a.force))
    except subprocess.CalledProcessError as e:
        sys.exit(e.returncode)
