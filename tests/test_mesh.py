"""The mesh builder (C library, isw.grid.build): from the reference's own smoothed positions it reproduces every integer
table of the reference grid bit for bit (numbering, neighbours, edges, Hilbert permutation, vertices, CSR, gather
orders) and its geometry to rounding; a full build passes the reference's GRID identities
(reference tests/test_grid.py:14-67)."""
import math

import numpy as np
import pytest
import torch

from conftest import GOLDEN

INTS = ('nbr', 'deg', 'eI', 'eJ', 'eKi', 'eKj', 'perm', 'cellEdge', 'cellSign', 'cellEdgeAsc', 'ev1', 'ev2', 'vEdge',
        'vEdgeSign', 'vCell', 'vSlot', 'eoeStart', 'eoe', 'cornerV', 'circ1', 'circ2')
FLOATS = ('pos', 'lat', 'lon', 'area', 'dist', 'edgeLen', 'le', 'de', 'areaCell', 'areaV', 'kite', 'w', 'fV', 'xm', 'ne', 'vPos')
SPHERE = 4 * math.pi * 6.371e6 ** 2


def identities(g):
    """Topology, areas, orthogonality, TRiSK antisymmetry and curl(grad) (reference tests/test_grid.py:14-57)."""
    n = g.n
    pent = int(np.sum(g.deg == 5))
    topo = bool(g.N == 10 * 4 ** n + 2 and g.E == 30 * 4 ** n and g.NV == 20 * 4 ** n and pent == 12
                and pent + int(np.sum(g.deg == 6)) == g.N and g.N - g.E + g.NV == 2
                and np.all(np.bincount(g.cellEdge[g.cellEdge >= 0], minlength=g.E) == 2)
                and np.all(np.bincount(g.cornerV[g.cornerV >= 0], minlength=g.NV) == 3))
    sums = max(abs(np.sum(a) - SPHERE) / SPHERE for a in (g.area, g.areaCell, g.areaV))
    kites = float(np.max(np.abs(g.areaCell - g.area) / g.area))
    t, d = g.vPos[g.ev2] - g.vPos[g.ev1], g.pos[g.eJ] - g.pos[g.eI]
    orth = float(np.max(np.abs(np.sum(t * d, axis=1)) / (np.linalg.norm(t, axis=1) * np.linalg.norm(d, axis=1))))
    e = np.repeat(np.arange(g.E, dtype=np.int64), np.diff(g.eoeStart))
    e2 = g.eoe.astype(np.int64)
    lhs = g.le[e] * g.de[e] * g.w
    key, rkey = e * g.E + e2, e2 * g.E + e
    o = np.argsort(key)
    j = o[np.searchsorted(key[o], rkey)]
    assert np.array_equal(key[j], rkey)
    anti = float(np.max(np.abs(lhs + lhs[j])) / np.max(np.abs(lhs)))
    f = 1e3 * np.sin(2 * g.lat) * np.cos(3 * g.lon) + 50 * g.pos[:, 0]
    gr = (f[g.eJ] - f[g.eI]) / g.de
    t1, t2 = g.circ1 * g.de * gr, g.circ2 * g.de * gr
    curl, mag = np.zeros(g.NV), np.zeros(g.NV)
    np.add.at(curl, g.ev1, t1)
    np.add.at(curl, g.ev2, t2)
    np.add.at(mag, g.ev1, np.abs(t1))
    np.add.at(mag, g.ev2, np.abs(t2))
    return topo, max(sums, kites, orth, anti, float(np.max(np.abs(curl) / mag)))


def test_tables_bit_exact_from_reference_positions(grid4):
    """Given the reference's smoothed level-4 positions, every integer table equals the reference's; geometry <= 1e-15."""
    from isw import grid as G
    v1 = np.empty_like(grid4.pos)
    v1[grid4.perm] = grid4.pos
    g = G.build(4, pos_v1=v1, device='cpu')
    for k in INTS:
        a, b = np.asarray(getattr(g, k)), np.asarray(getattr(grid4, k))
        assert a.shape == b.shape and np.array_equal(a, b), k
    for k in FLOATS:
        a, b = np.asarray(getattr(g, k), dtype=float), np.asarray(getattr(grid4, k), dtype=float)
        assert np.max(np.abs(a - b)) <= 1e-15 * np.max(np.abs(b)), k


def test_hilbert_order_matches_reference(grid4):
    """The 21-bit 3-D Hilbert key order of the v1 positions is the reference's permutation."""
    from isw import grid as G
    v1 = np.empty_like(grid4.pos)
    v1[grid4.perm] = grid4.pos
    g = G.build(4, pos_v1=v1, device='cpu', order='hilbert')
    assert np.array_equal(g.perm, grid4.perm)
    gv = G.build(4, pos_v1=v1, device='cpu', order='v1')
    assert np.array_equal(gv.pos, v1)          # v1 numbering: the icosphere's own
    assert gv.E == grid4.E and gv.NV == grid4.NV


@pytest.mark.parametrize('n', [0, 1, 2, 3])
def test_full_build_identities(n):
    """Icosphere + Lloyd on host cores + tables: the reference's GRID identities hold (topology exact, <= 1e-12)."""
    from isw import grid as G
    g = G.build(n, device='cpu')
    topo, worst = identities(g)
    assert topo and worst <= 1e-12, worst


def test_full_build_level4_matches_reference_lloyd(grid4):
    """A full level-4 build takes the reference's number of Lloyd iterations and lands on its positions to rounding."""
    from isw import grid as G
    g = G.build(4, device='cpu')
    assert g.lloydIters == int(grid4.lloydIters)
    assert np.max(np.abs(g.pos - grid4.pos)) <= 1e-14
    topo, worst = identities(g)
    assert topo and worst <= 1e-12


@pytest.mark.gpu
def test_gpu_lloyd(grid4):
    """Lloyd on the GPU: level 4 converges like the reference (iterations within one, positions to 1e-13); level 6
    builds and passes the GRID identities."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from isw import grid as G
    g = G.build(4, device=0)
    assert abs(g.lloydIters - int(grid4.lloydIters)) <= 1
    assert np.max(np.abs(g.pos - grid4.pos)) <= 1e-13
    g6 = G.build(6, device=0)
    topo, worst = identities(g6)
    assert topo and worst <= 1e-12


def _reference_grid6():
    from oracle import build_ref
    p = build_ref.grid_path(6)
    if not p.exists():
        pytest.skip('the reference-built level-6 grid (oracle/_ref) is not present')
    from isw import grid as G
    return G.load(p)


def test_level6_tables_bit_exact_from_reference_positions():
    """Level 6: from the positions the reference's own Lloyd iteration gave (tests/golden/pos_n6.npz), the mesh
    builder reproduces every integer table of the grid the reference's own Python builds from them (oracle/_ref,
    oracle/build_ref.py) bit for bit, and its geometry to 1e-14."""
    from isw import grid as G
    ref = _reference_grid6()
    with np.load(GOLDEN / 'pos_n6.npz') as z:
        v1 = z['pos']
        assert int(z['lloydIters']) == int(ref.lloydIters)
    g = G.build(6, pos_v1=v1, device='cpu')
    for k in INTS:
        a, b = np.asarray(getattr(g, k)), np.asarray(getattr(ref, k))
        assert a.shape == b.shape and np.array_equal(a, b), k
    for k in FLOATS:
        a, b = np.asarray(getattr(g, k), dtype=float), np.asarray(getattr(ref, k), dtype=float)
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b)), k


def test_full_build_level6_lloyd_matches_reference():
    """A full level-6 build on the host cores takes the reference's Lloyd iteration count (5412) and lands on its
    positions to rounding."""
    from isw import grid as G
    with np.load(GOLDEN / 'pos_n6.npz') as z:
        v1, iters = z['pos'], int(z['lloydIters'])
    g = G.build(6, order='v1', device='cpu')
    assert g.lloydIters == iters
    assert np.max(np.abs(g.pos - v1)) <= 1e-13
