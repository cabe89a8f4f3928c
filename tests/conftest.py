"""Shared test set-up: import paths, the `gpu` marker, fixture loaders."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / 'insilica-world-v2_b200'
GOLDEN = Path(__file__).resolve().parent / 'golden'
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200); run with -m gpu')


def _ensure_oracle():
    lib = ROOT / 'oracle' / 'liboracle.so'
    src = ROOT / 'oracle' / 'oracle.c'
    if not lib.exists() or lib.stat().st_mtime < src.stat().st_mtime:
        from oracle import model
        model.build()


@pytest.fixture(scope='session')
def oracle_lib():
    _ensure_oracle()
    from oracle import model
    return model


def golden(name):
    with np.load(GOLDEN / f'{name}.npz') as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope='session')
def grid4():
    from isw import grid as G
    return G.load(GOLDEN / 'grid_n4.npz')
