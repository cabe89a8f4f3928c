"""ctypes driver for ``oracle/_ref/libref_kernels.so``: the reference's own kernels compiled as host C++.

TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; never part of the product path).

``RefKernels().launch(name, grid, block, args)`` takes the same arguments the reference passes to a CuPy
``RawKernel`` (``grid=(gx, gy)``, ``block=(bx,)``, ``args`` a tuple of NumPy scalars and C-contiguous NumPy arrays, or
``0`` for a null pointer) and runs the kernel over that grid on the host.
"""
import ctypes
import json
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / '_ref'
_CT = {'int': ctypes.c_int, 'i64': ctypes.c_longlong, 'real': ctypes.c_double, 'f32': ctypes.c_float,
       'f64': ctypes.c_double, 'ptr': ctypes.c_void_p}


def available():
    return (REF_DIR / 'libref_kernels.so').exists() and (REF_DIR / 'ref_kernels.json').exists()


class RefKernels:
    def __init__(self, path=REF_DIR):
        path = Path(path)
        self.lib = ctypes.CDLL(str(path / 'libref_kernels.so'))
        self.sigs = json.loads((path / 'ref_kernels.json').read_text())
        self._fn = {}
        for name, s in self.sigs.items():
            f = getattr(self.lib, f'ref_{name}')
            f.restype = None
            f.argtypes = [ctypes.c_int] * 3 + [_CT[p[2]] for p in s['params']]
            self._fn[name] = (f, [p[2] for p in s['params']])

    def has(self, name):
        return name in self._fn

    def launch(self, name, grid, block, args):
        f, kinds = self._fn[name]
        if len(args) != len(kinds):
            raise TypeError(f'{name}: {len(args)} arguments, kernel takes {len(kinds)}')
        gx, gy = (tuple(grid) + (1,))[:2]
        conv = []
        keep = []
        for a, k in zip(args, kinds):
            if k == 'ptr':
                if isinstance(a, np.ndarray):
                    if not a.flags.c_contiguous:
                        raise ValueError(f'{name}: non-contiguous array argument')
                    keep.append(a)
                    conv.append(ctypes.c_void_p(a.ctypes.data))
                else:
                    if int(a) != 0:
                        raise ValueError(f'{name}: pointer argument must be an array or 0')
                    conv.append(ctypes.c_void_p(None))
            elif k in ('int', 'i64'):
                conv.append(int(a))
            else:
                conv.append(float(a))
        f(int(gx), int(gy), int(block[0]), *conv)
