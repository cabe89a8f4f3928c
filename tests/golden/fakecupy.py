"""A NumPy-backed stand-in for the parts of CuPy that the reference's ``gpu.py``, ``layers.py`` and
``transport.py`` use, so those modules run UNCHANGED on the host to generate golden vectors.

Used only by ``tests/golden/make_golden.py`` in a container that holds the reference sources; never by the product.

- Device arrays are NumPy arrays (``DevArray`` adds CuPy's ``.get()``).
- ``RawModule(code=..., options=...)`` finds which reference kernel file the source is (by its kernel names) and
  returns functions that run the host-compiled reference kernels from ``oracle/_ref`` (``oracle/refkernels.py``).
  Only the FP64 form (``-DREAL=double`` without ``-DMIXED``) is supported.
- ``block_sum`` (reference ``kernels/trisk.cu:61-81``) is a shared-memory tree: it runs here as the same fixed tree
  in NumPy (thread t sums its 8 strided values in order, then the 256 partial sums halve pairwise).
"""
import re
import sys
import types
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from oracle.refkernels import RefKernels  # noqa: E402

float64, float32, int32, int8, uint64 = np.float64, np.float32, np.int32, np.int8, np.uint64
_K = None


class DevArray(np.ndarray):
    def get(self):
        return np.array(self)


def _dev(a):
    a = np.ascontiguousarray(a)
    return a.view(DevArray)


def asarray(a, dtype=None):
    return _dev(np.array(a, dtype=dtype, copy=True))


def ascontiguousarray(a):
    return _dev(np.ascontiguousarray(a))


def zeros(shape, dtype=float):
    return _dev(np.zeros(shape, dtype=dtype))


def empty(shape, dtype=float):
    return _dev(np.zeros(shape, dtype=dtype))


def full(shape, value, dtype=None):
    return _dev(np.full(shape, value, dtype=dtype))


def zeros_like(a):
    return _dev(np.zeros_like(a))


def copyto(dst, src, casting='same_kind'):
    np.copyto(dst, np.asarray(src), casting=casting)


max, sum, min, abs, all, isfinite = np.max, np.sum, np.min, np.abs, np.all, np.isfinite
linalg = types.SimpleNamespace(norm=np.linalg.norm)


def _block_sum_tree(n, x, y, out):
    threads, chunk = 256, 8
    n = int(n)
    xv = np.asarray(x)[:n]
    v = xv * np.asarray(y)[:n] if not isinstance(y, (int, np.integer)) else xv.copy()
    blocks = len(out)
    per = threads * chunk
    pad = np.zeros(blocks * per, dtype=v.dtype)
    pad[:n] = v
    pad = pad.reshape(blocks, chunk, threads)
    acc = np.zeros((blocks, threads), dtype=v.dtype)
    for k in range(chunk):               # acc += x[base + t + 256 k], k ascending (zeros past n add exactly 0)
        acc = acc + pad[:, k, :]
    h = threads // 2
    while h > 0:
        acc[:, :h] = acc[:, :h] + acc[:, h:2 * h]
        h //= 2
    out[:] = acc[:, 0]


class _Function:
    def __init__(self, name):
        self.name = name

    def __call__(self, grid, block, args):
        if self.name == 'block_sum':
            return _block_sum_tree(*args)
        _K.launch(self.name, grid, block, args)


class RawModule:
    def __init__(self, code, options=()):
        global _K
        if any('MIXED' in o for o in options):
            raise NotImplementedError('the stand-in runs the FP64 reference only')
        if not any(o == '-DREAL=double' for o in options):
            raise NotImplementedError('the stand-in runs REAL=double only')
        if _K is None:
            _K = RefKernels()
        self.names = set(re.findall(r'__global__\s+void\s+(\w+)', code))

    def get_function(self, name):
        if name not in self.names:
            raise KeyError(name)
        return _Function(name)


class _Stream:
    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def synchronize(self):
        pass


cuda = types.SimpleNamespace(Stream=_Stream)


def install():
    """Make ``import cupy`` return this module."""
    sys.modules['cupy'] = sys.modules[__name__]
