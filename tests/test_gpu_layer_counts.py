"""Layer and tracer counts the golden cases do not reach (1, 5 and 8 layers; 1 to 16 tracers), against the oracle
(oracle/model.py over the C restatement), bit for bit: the FCT fields are stored with an item's layers side by side,
padded to an even count, so odd counts and the largest count take their own load and store paths. No stress terms,
so no exp() enters and the FP64 form must match exactly.
  - Transport.step_many call by call, orders 1 and 3
  - the batched step (dynamics, receiving masses and FCT of every stack in one graph) at 5 and 8 layers, tiled and
    grid-wide
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda:0')


def _T(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


def _masses_and_fluxes(grid, L, seed):
    """Layer masses of ~300 m layers and a random edge flux small enough that no cell empties."""
    rng = np.random.default_rng(seed)
    h = 300.0 + 20.0 * rng.random((L, grid.N))
    M0 = h * np.asarray(grid.areaCell)[None]
    Fm = 2e-3 * float(M0.min()) * (rng.random((L, grid.E)) - 0.5)
    return M0, Fm


@pytest.mark.parametrize('L,ntr', [(1, 16), (5, 3), (8, 2)])
@pytest.mark.parametrize('order', [1, 3])
def test_transport_layer_counts(dev, grid4, oracle_lib, L, ntr, order):
    from isw import gpu, transport
    gpu.set_precision('double')
    O = oracle_lib
    dg, og = gpu.DeviceGrid(grid4), O.OracleGrid(grid4)
    tr, otr = transport.Transport(dg, layers=L, tracers=ntr), O.Transport(og, layers=L, tracers=ntr)
    M0, Fm = _masses_and_fluxes(grid4, L, 10 * L + ntr)
    rng = np.random.default_rng(L * 100 + ntr)
    psi = [rng.random((L, grid4.N)) + 0.5 * k for k in range(ntr)]
    gM, gM1, gF = _T(M0, dev), torch.zeros(L, grid4.N, dtype=torch.float64, device=dev), _T(Fm, dev)
    gpsi = [_T(p, dev) for p in psi]
    oM, oM1 = M0.copy(), np.zeros_like(M0)
    for _ in range(3):
        tr.mass_after(gM, gF, gM1)
        tr.step_many(gM, gM1, gF, gpsi, order=order)
        gM, gM1 = gM1, gM
        otr.mass_after(oM, Fm, oM1)
        otr.step_many(oM, oM1, Fm, psi, order=order)
        oM, oM1 = oM1, oM
    torch.cuda.synchronize()
    assert np.array_equal(gM.cpu().numpy(), oM)
    for k in range(ntr):
        assert np.array_equal(gpsi[k].cpu().numpy(), psi[k]), k


@pytest.mark.parametrize('L', [5, 8])
@pytest.mark.parametrize('tiles', [True, False])
def test_batched_step_layer_counts(dev, grid4, oracle_lib, L, tiles):
    """One stack of L layers with 2 tracers, 3 batched steps (nabla^4, drag, 4 fast sub-steps per stage) against the
    oracle's Layers.step + mass_after + step_many, bit for bit in h, u, Fm, M and the tracers."""
    from isw import gpu, transport
    from isw.batch import Batch
    from isw.layers import Layers
    gpu.set_precision('double')
    O = oracle_lib
    dg, og = gpu.DeviceGrid(grid4), O.OracleGrid(grid4)
    rng = np.random.default_rng(L)
    N, E = grid4.N, grid4.E
    h0 = 300.0 + 10.0 * rng.random((L, N))
    b = -300.0 * L + 50.0 * rng.random(N)
    u0 = 0.5 * (rng.random((L, E)) - 0.5)
    psi = [rng.random((L, N)), 1.0 + rng.random((L, N))]
    kw = dict(b=b, gprime=[0.05] * (L - 1), drag=1e-6, nu4=1e14)
    dt, nfast = 900.0, 4
    core, tr = Layers(dg, L, **kw), transport.Transport(dg, layers=L, tracers=2)
    oc, otr = O.Layers(og, L, **kw), O.Transport(og, layers=L, tracers=2)
    h, u, Fm = _T(h0, dev), _T(u0, dev), torch.zeros(L, E, dtype=torch.float64, device=dev)
    M = _T(h0 * np.asarray(grid4.areaCell)[None], dev)
    M1 = torch.zeros_like(M)
    gpsi = [_T(p, dev) for p in psi]
    batch = Batch(0)
    batch.config(tiles=tiles)
    batch.add(core, h, u, Fm, tr=tr, M=M, M1=M1, tracers=gpsi, dt=dt, nfast=nfast)
    oh, ou, oF = h0.copy(), u0.copy(), np.zeros((L, E))
    oM, oM1 = h0 * np.asarray(grid4.areaCell)[None], np.zeros((L, N))
    for _ in range(3):
        batch.step()
        oc.step(oh, ou, dt, nfast, oF)
        otr.mass_after(oM, oF, oM1)
        otr.step_many(oM, oM1, oF, psi)
        oM, oM1 = oM1, oM
    torch.cuda.synchronize()
    assert batch.status() == 0
    assert (batch.info()['tiles'] > 0) == tiles
    for name, a, ref in (('h', h, oh), ('u', u, ou), ('Fm', Fm, oF), ('M', M, oM), ('tr0', gpsi[0], psi[0]),
                         ('tr1', gpsi[1], psi[1])):
        assert np.array_equal(a.cpu().numpy(), ref), name
