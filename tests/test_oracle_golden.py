"""The oracle pinned to the reference: the C restatement (oracle/oracle.c), its single-process NumPy form
(oracle/numpy_kernels.py) and the host-compiled reference kernels (oracle/_ref), all driven by oracle/model.py,
reproduce the golden vectors the reference's own Python produced (tests/golden/make_golden.py) bit for bit. CPU only."""
import numpy as np
import pytest

from conftest import golden
from oracle import refkernels

BACKENDS = ['oracle', 'numpy'] + (['reference'] if refkernels.available() else [])


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _grid(grid4, omega=None):
    from isw import grid as G
    return G.for_planet(grid4, 6.371e6, omega, 9.80616) if omega else grid4


@pytest.mark.parametrize('backend', BACKENDS)
def test_w2_bit_exact(oracle_lib, grid4, backend):
    """Williamson 2 (n = 4, dt 900 s): 1, 96, 480 steps equal the reference's bit for bit; energy too."""
    M = oracle_lib
    z = golden('w2_n4')
    dg = M.OracleGrid(_grid(grid4, float(z['omega'])))
    core = M.Layers(dg, 1, b=z['b'], backend=backend)
    h, u = z['h0'].copy(), z['u0'].copy()
    assert core.substeps(h, float(z['dt'])) == int(z['substeps'])
    assert core.energy(h, u) == float(z['energy0'])
    for s in range(1, 481):
        core.step(h, u, float(z['dt']), int(z['nfast']))
        if s in (1, 96, 480):
            assert np.array_equal(h, z[f'h{s}']) and np.array_equal(u, z[f'u{s}']), s
    assert core.energy(h, u) == float(z['energy480'])


def run_stack(M, grid4, z, backend, steps):
    dg = M.OracleGrid(_grid(grid4, 7.292e-5))
    L = int(z['L'])
    core = M.Layers(dg, L, b=z['b'], gprime=list(z['gprime']), stress=list(z['stress']), nu4=float(z['nu4']),
                    floor=float(z['floor']), vmix=float(z['vmix']), backend=backend)
    tr = M.Transport(dg, layers=L, tracers=3, backend=backend)
    h, u = z['h0'].copy(), z['u0'].copy()
    Mm = z['h0'] * dg.host.areaCell[None]
    trc = [z[f'tr{k}_0'].copy() for k in range(3)]
    Fm, M1 = np.zeros((L, dg.E)), np.zeros((L, dg.N))
    out = {}
    for st in range(1, steps + 1):
        core.step(h, u, float(z['dt']), int(z['nfast']), Fm)
        tr.mass_after(Mm, Fm, M1)
        tr.step_many(Mm, M1, Fm, trc, order=3)
        Mm, M1 = M1, Mm
        if st == 1:
            out['h1'], out['u1'], out['M1'], out['tr1'] = h.copy(), u.copy(), Mm.copy(), [t.copy() for t in trc]
    return core, h, u, Mm, trc, Fm, out


@pytest.mark.parametrize('backend', BACKENDS)
@pytest.mark.parametrize('case', ['air3_n4', 'ocean2_n4'])
def test_stacks_bit_exact(oracle_lib, grid4, backend, case):
    """Stacked layers with nu4, stress, interfacial stress, 20 fast sub-steps and 3 FCT tracers: every array equal."""
    import hashlib
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    z = golden(case)
    core, h, u, Mm, trc, Fm, one = run_stack(oracle_lib, grid4, z, backend, 6)
    assert abs(core.lap_max() - float(z['lap_max'])) <= 1e-12 * float(z['lap_max'])
    if backend == 'numpy':              # NumPy's exp (the stress terms) may round the last bit differently from libm's
        for name, a in (('h', h), ('u', u), ('M', Mm), ('Fm', Fm)) + tuple((f'tr{k}', trc[k]) for k in range(3)):
            assert rel(a, z[name]) <= 1e-13, name
        return
    assert sha(one['h1']) == str(z['sha_h1']) and sha(one['u1']) == str(z['sha_u1']) and sha(one['M1']) == str(z['sha_M1'])
    for k in range(3):
        assert sha(one['tr1'][k]) == str(z[f'sha_tr{k}_1'])
    for name, a in (('h', h), ('u', u), ('M', Mm), ('Fm', Fm)):
        assert np.array_equal(a, z[name]), name
    for k in range(3):
        assert np.array_equal(trc[k], z[f'tr{k}']), k


@pytest.mark.parametrize('backend', BACKENDS)
def test_outcrop_bit_exact(oracle_lib, grid4, backend):
    """The reference's outcrop case (floor limiter active, bottom stress, nu4) with the bell tracer, 24 steps."""
    M = oracle_lib
    z = golden('outcrop_n4')
    dg = M.OracleGrid(grid4)
    core = M.Layers(dg, 2, b=z['b'], gprime=[0.02], stress=[0.0, 2.5e-4], nu4=float(z['nu4']), floor=1.0, backend=backend)
    tr = M.Transport(dg, layers=2, tracers=4, backend=backend)
    h, u, psi = z['h0'].copy(), z['u0'].copy(), z['psi0'].copy()
    assert core.substeps(h, float(z['dt'])) * 1.2 <= int(z['nfast'])
    Mm = z['h0'] * grid4.areaCell[None]
    Fm, M1 = np.zeros((2, dg.E)), np.zeros((2, dg.N))
    lo = float(h.min())
    for _ in range(24):
        core.step(h, u, float(z['dt']), int(z['nfast']), Fm)
        tr.mass_after(Mm, Fm, M1)
        tr.step_many(Mm, M1, Fm, [psi], order=3)
        Mm, M1 = M1, Mm
        lo = min(lo, float(h.min()))
    for name, a in (('h', h), ('u', u), ('M', Mm), ('psi', psi), ('Fm', Fm)):
        if backend == 'numpy':          # its exp (the bottom stress) may differ from libm's in the last bit
            assert rel(a, z[name]) <= 1e-12, name
        else:
            assert np.array_equal(a, z[name]), name
    assert lo == float(z['hmin']) or (backend == 'numpy' and abs(lo - float(z['hmin'])) <= 1e-12 * abs(lo))


@pytest.mark.parametrize('backend', BACKENDS)
def test_bell_bit_exact(oracle_lib, grid4, backend):
    """Transport alone (the cosine bell in solid-body rotation), order 1 and order 3, 20 steps."""
    M = oracle_lib
    z = golden('bell_n4')
    dg = M.OracleGrid(grid4)
    for order in (1, 3):
        tr = M.Transport(dg, backend=backend)
        psi, Mb, Mb1 = z['psi0'].copy(), z['M0'].copy(), np.zeros((1, dg.N))
        for _ in range(20):
            tr.mass_after(Mb, z['Fm'], Mb1)
            tr.step(Mb, Mb1, z['Fm'], psi, order)
            Mb, Mb1 = Mb1, Mb
        assert np.array_equal(psi, z[f'psi_o{order}']) and np.array_equal(Mb, z[f'M_o{order}'])


def test_dsum_tree(oracle_lib):
    """The deterministic tree sum equals the reference's block_sum passes bit for bit."""
    z = golden('dsum')
    for n in (1, 2, 255, 2048, 2049, 100003, 1 << 20):
        i = np.arange(n, dtype=np.int64)
        x = ((i * 7919) % 10007 - 5003) / 997.0
        y = ((i * 104729) % 65521) / 4093.0
        assert oracle_lib.dsum(x) == float(z[f'x_{n}'])
        assert oracle_lib.dsum(x, y) == float(z[f'xy_{n}'])
        assert oracle_lib.dsum(x, backend='numpy') == float(z[f'x_{n}'])
        assert oracle_lib.dsum(x, y, backend='numpy') == float(z[f'xy_{n}'])


def test_d2_stencil_matches_reference_formula(oracle_lib, grid4):
    """d2_stencil: indices are cells of the edge's two ends and their opposite neighbours; weights sum to zero."""
    idx, wt = oracle_lib.d2_stencil(grid4)
    idx = idx.reshape(-1, 2, 4)
    assert np.array_equal(idx[:, 0, 0], grid4.eI) and np.array_equal(idx[:, 1, 0], grid4.eJ)
    assert np.array_equal(idx[:, 0, 1], grid4.eJ) and np.array_equal(idx[:, 1, 1], grid4.eI)
    s = wt.reshape(-1, 2, 4).sum(axis=2)
    assert np.max(np.abs(s)) <= 1e-9 * np.max(np.abs(wt))
