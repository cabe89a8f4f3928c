"""Oracle driver: the reference's ``Layers.step`` / ``Transport.step_many`` / ``DeviceGrid`` / ``dsum`` restated in
NumPy + ctypes over a kernel backend.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``,
never by the product.

Backends (the same kernel argument lists, so one driver runs them all):
- ``'oracle'``: this project's plain-C restatement ``oracle/oracle.c`` (``liboracle.so``, OpenMP),
- ``'reference'``: the reference's own kernels compiled for the host (``oracle/_ref``, see ``build_ref.py``),
- ``'numpy'``: the same kernels as whole-array NumPy operations in one process (``oracle/numpy_kernels.py``).

The driver follows the reference call sequence line by line:
- ``Layers.__init__``  reference ``src/insilica/layers.py:36-92`` (Boussinesq options: gprime, drag, stress, nu4, floor,
  rotation, div_damp, thin, vmix, vmix_cd; the air, wall, shelf, sig, tide options are refused)
- ``Layers.substeps``  ``layers.py:99-102``;  ``lap_max`` ``:111-121``;  ``_lap`` ``:123-127``
- ``Layers._stage``    ``layers.py:129-183`` (Boussinesq branch, ``:137-140`` and ``:167-183``)
- ``Layers.step``      ``layers.py:185-212``;  ``energy`` ``:234-253`` (Boussinesq form)
- ``Transport``        ``transport.py:18-71``
- ``d2_stencil``       ``gpu.py:86-108``;  ``dsum`` ``gpu.py:111-126`` (the tree in ``oracle.c``)
"""
import ctypes
import math
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LMAX = 8
FAST_COURANT = 0.5
DIV_DAMP = 0.1
BETA = 0.25
BLOCK = 64

_CT = {'int': ctypes.c_int, 'i64': ctypes.c_longlong, 'real': ctypes.c_double, 'ptr': ctypes.c_void_p}


def _kind(t):
    if '*' in t:
        return 'ptr'
    t = t.replace('const', '').strip()
    return {'int': 'int', 'long long': 'i64', 'real': 'real', 'double': 'real'}[t]


class OracleKernels:
    """ctypes binding of oracle/liboracle.so; signatures read from oracle.c itself."""

    def __init__(self, lib=HERE / 'liboracle.so', src=HERE / 'oracle.c'):
        self.lib = ctypes.CDLL(str(lib))
        text = Path(src).read_text()
        self.sig = {}
        for m in re.finditer(r'^(?:void|real)\s+o_(\w+)\s*\(([^)]*)\)\s*\{', text, re.M | re.S):
            kinds = []
            for p in m.group(2).split(','):
                p = ' '.join(p.split())
                name = re.findall(r'(\w+)\s*$', p)[0]
                kinds.append(_kind(p[: len(p) - len(name)]))
            f = getattr(self.lib, f'o_{m.group(1)}')
            f.argtypes = [_CT[k] for k in kinds]
            self.sig[m.group(1)] = (f, kinds)
        self.sig['dsum'][0].restype = ctypes.c_double
        self.lib.o_error.restype = ctypes.c_int

    def __call__(self, name, n, rows, args):
        f, kinds = self.sig[name]
        f(*_convert(name, (rows,) + tuple(args), kinds))
        if self.lib.o_error():
            raise NotImplementedError(f'oracle {name}: option branch not restated')

    def dsum(self, x, y=None):
        f, kinds = self.sig['dsum']
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = None if y is None else np.ascontiguousarray(y, dtype=np.float64).ravel()
        return float(f(*_convert('dsum', (x.size, x, y), kinds)))


class ReferenceKernels:
    """The reference's own kernels on the host (oracle/_ref)."""

    def __init__(self):
        from oracle.refkernels import RefKernels
        self.k = RefKernels()
        self._ora = None

    def __call__(self, name, n, rows, args):
        self.k.launch(name, ((n + BLOCK - 1) // BLOCK, rows), (BLOCK,), tuple(0 if a is None else a for a in args))

    def dsum(self, x, y=None):          # block_sum is not a per-thread kernel: the oracle's restatement of its tree
        if self._ora is None:
            self._ora = OracleKernels()
        return self._ora.dsum(x, y)


def _convert(name, args, kinds):
    if len(args) != len(kinds):
        raise TypeError(f'{name}: {len(args)} arguments for {len(kinds)} parameters')
    out = []
    for a, k in zip(args, kinds):
        if k == 'ptr':
            if a is None:
                out.append(None)
            else:
                if not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
                    raise TypeError(f'{name}: pointer argument must be a C-contiguous array')
                out.append(a.ctypes.data)
        elif k in ('int', 'i64'):
            out.append(int(a))
        else:
            out.append(float(a))
    return out


_BACKENDS = {}


def kernels(backend='oracle'):
    if backend not in _BACKENDS:
        if backend == 'numpy':
            from oracle.numpy_kernels import NumpyKernels
            _BACKENDS[backend] = NumpyKernels()
        else:
            _BACKENDS[backend] = OracleKernels() if backend == 'oracle' else ReferenceKernels()
    return _BACKENDS[backend]


def d2_stencil(g):
    """Per edge end, weights on four cells for the 3rd-order transport's second derivative (reference gpu.py:86-108)."""
    E = g.E
    nbr, deg, dist = g.nbr.astype(np.int64), g.deg.astype(np.int64), g.dist
    idx = np.zeros((E, 2, 4), dtype=np.int32)
    wt = np.zeros((E, 2, 4))
    for side, (c, k) in enumerate(((g.eI.astype(np.int64), g.eKi.astype(np.int64)), (g.eJ.astype(np.int64), g.eKj.astype(np.int64)))):
        m = deg[c]
        j = nbr[c, k]
        d1 = dist[c, k]
        hexa = m == 6
        ka = np.where(hexa, (k + 3) % 6, (k + 2) % m)
        kb = np.where(hexa, (k + 3) % 6, (k + 3) % m)
        o1, o2 = nbr[c, ka], nbr[c, kb]
        d2v = np.where(hexa, dist[c, (k + 3) % 6], 0.5 * (dist[c, ka] + dist[c, kb]))
        s = 2 / (d1 + d2v) * g.de * g.de / 12
        idx[:, side] = np.stack([c, j, o1, o2], axis=1)
        wt[:, side, 0] = -s * (1 / d1 + 1 / d2v)
        wt[:, side, 1] = s / d1
        wt[:, side, 2] = 0.5 * s / d2v
        wt[:, side, 3] = 0.5 * s / d2v
    return idx.reshape(-1), wt.reshape(-1)


class OracleGrid:
    """A grid's arrays typed as the reference's DeviceGrid holds them in its FP64 form (reference gpu.py:55-83)."""
    INT32 = ('eI', 'eJ', 'nbr', 'cellEdge', 'cellEdgeAsc', 'ev1', 'ev2', 'vEdge', 'vCell', 'eoeStart', 'eoe')
    INT8 = ('cellSign', 'vEdgeSign', 'vSlot')
    REALS = ('le', 'de', 'areaCell', 'areaV', 'fV', 'kite', 'w')

    def __init__(self, grid):
        self.host = grid
        self.n, self.N, self.E, self.NV = int(grid.n), int(grid.N), int(grid.E), int(grid.NV)
        for k in self.INT32:
            setattr(self, k, np.ascontiguousarray(getattr(grid, k), dtype=np.int32))
        for k in self.INT8:
            setattr(self, k, np.ascontiguousarray(getattr(grid, k), dtype=np.int8))
        for k in self.REALS:
            setattr(self, k, np.ascontiguousarray(getattr(grid, k), dtype=np.float64))
        self.d2idx, self.d2wt = d2_stencil(grid)
        self.d2wt_tr = self.d2wt
        self.rA, self.rde, self.rAV = self.areaCell, self.de, self.areaV


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Layers:
    def __init__(self, dg, layers=1, b=None, grav=9.80616, gprime=(), drag=0.0, stress=0.0, nu4=0.0, floor=1.0, rotation=1.0,
                 div_damp=DIV_DAMP, thin=2.0, vmix=0.0, vmix_cd=0.0, backend='oracle'):
        assert 1 <= layers <= LMAX and len(gprime) == layers - 1
        self.K = kernels(backend)
        self.dg, self.L = dg, layers
        self.grav, self.nu4, self.floor, self.div_damp, self.thin = grav, nu4, floor, div_damp, thin
        self.vmix, self.vmix_cd = vmix, vmix_cd
        N, E, NV, L = dg.N, dg.E, dg.NV, layers
        z = lambda *s: np.zeros(s)
        self.b = z(N) if b is None else _c(b).copy()
        self.gp = _c(np.asarray(gprime, dtype=float).reshape(-1) if layers > 1 else np.zeros(1))
        self.drag = _c(np.broadcast_to(np.asarray(drag, dtype=float), (layers,)))
        self.stress = _c(np.broadcast_to(np.asarray(stress, dtype=float), (layers,)))
        self.fV = dg.fV * rotation
        self.Gc = np.full(N, float(grav))
        self.B, self.q, self.Tp, self.F, self.scale = z(L, N), z(L, NV), z(L, E), z(L, E), z(L, N)
        self.G, self.He, self.ubs, self.ub0, self.ub, self.acc = z(E), z(E), z(E), z(E), z(E), z(E)
        self.eta0, self.eta, self.eta_prev = z(N), z(N), z(N)
        self.h1, self.h2, self.u1, self.u2 = z(L, N), z(L, N), z(L, E), z(L, E)
        self.D1, self.Z1, self.L1, self.L2 = z(L, N), z(L, NV), z(L, E), z(L, E)
        self.hedge, self.diss = z(L, E), z(E)
        self.pk = np.zeros(3 * L * E)
        self.wf = dg.w
        self.dmin = float(np.min(dg.host.de))

    def substeps(self, h, dt):
        c2 = float(np.max(np.sum(h, axis=0) * self.Gc))
        return max(1, math.ceil(dt * math.sqrt(c2) / (FAST_COURANT * self.dmin)))

    def lap_max(self, iters=30):
        v = np.random.default_rng(0).standard_normal((self.L, self.dg.E))
        lam = 0.0
        for _ in range(iters):
            self._lap(v, self.L1)
            lam = float(np.linalg.norm(self.L1[0]) / np.linalg.norm(v[0]))
            v = self.L1 / np.linalg.norm(self.L1[0])
        return lam

    def _lap(self, u, out):
        g, K, L = self.dg, self.K, self.L
        K('cell_div', g.N, L, (g.N, g.E, u, g.cellEdge, g.cellSign, g.le, g.areaCell, self.D1))
        K('vertex_curl', g.NV, L, (g.E, g.NV, u, g.vEdge, g.vEdgeSign, g.de, g.areaV, self.Z1))
        K('edge_lap', g.E, L, (g.N, g.E, g.NV, self.D1, self.Z1, g.eI, g.eJ, g.ev1, g.ev2, g.de, g.le, out))

    def _stage(self, hs, us, h0, u0, c, dt, nfast, hn, un, Fm=None):
        g, K, L = self.dg, self.K, self.L
        N, E, NV = g.N, g.E, g.NV
        K('lay_bern', N, 1, (N, E, L, hs, us, self.b, self.gp, g.cellEdge, g.le, g.de, g.areaCell, self.B, None, None, None))
        K('swe_vertex', NV, L, (N, E, NV, hs, us, g.vCell, g.vSlot, g.kite, g.vEdge, g.vEdgeSign, g.de, g.rAV, self.fV, self.q))
        K('lay_edge_hq', E, L, (N, E, NV, hs, self.q, g.eI, g.eJ, g.ev1, g.ev2, 0.0, us, self.hedge, self.pk, None))
        K('lay_slow', E, 1, (N, E, L, self.pk, self.wf, self.hedge, us, self.B, g.eoeStart, g.eoe, g.eI, g.eJ, g.rde,
                             self.drag, self.stress, self.floor, self.nu4, self.L2 if self.nu4 else None, None, None,
                             c * dt, self.thin, 0.0, self.Tp, self.G, self.He, self.ubs, None, None, None, 0.0, None))
        n = max(1, math.ceil(c * nfast))
        tau = c * dt / n
        np.copyto(self.eta, self.eta0)
        np.copyto(self.ub, self.ub0)
        self.acc.fill(0)
        for _ in range(n):
            K('bt_eta', N, 1, (N, self.He, self.ub, g.cellEdge, g.cellSign, g.le, g.rA, tau, self.eta, self.eta_prev))
            K('bt_u', E, 1, (E, self.eta, self.eta_prev, self.div_damp, self.G, g.eI, g.eJ, g.rde, self.Gc, tau, self.ub, self.acc))
        K('lay_flux', E, L, (N, E, hs, us, self.ubs, self.acc, 1.0 / n, g.eI, g.eJ, 0.0, self.F, None))
        K('lay_scale', N, L, (N, E, h0, self.F, g.cellEdgeAsc, g.eI, g.le, g.areaCell, c * dt, self.floor, self.scale))
        K('lay_limit', E, L, (N, E, g.eI, g.eJ, self.scale, g.le, dt, self.F, Fm))
        K('lay_h', N, L, (N, E, h0, self.F, g.cellEdge, g.cellSign, g.le, g.rA, c * dt, hn))
        K('lay_u', E, L, (E, u0, self.Tp, self.ub, self.ub0, c * dt, un))

    def step(self, h, u, dt, nfast, Fm=None):
        """One time-split RK3 step in place on h (L, N), u (L, E) (reference layers.py:185-212, Boussinesq branch)."""
        g, K, L = self.dg, self.K, self.L
        K('lay_eta', g.N, 1, (g.N, L, h, self.b, self.eta0))
        K('lay_ubar', g.E, 1, (g.N, g.E, L, h, u, g.eI, g.eJ, 0.0, self.ub0, None))
        if self.nu4:
            self._lap(u, self.L1)
            self._lap(self.L1, self.L2)
        self._stage(h, u, h, u, 1 / 3, dt, nfast, self.h1, self.u1)
        self._stage(self.h1, self.u1, h, u, 1 / 2, dt, nfast, self.h2, self.u2)
        self._stage(self.h2, self.u2, h, u, 1.0, dt, nfast, h, u, Fm)
        if (self.vmix or self.vmix_cd) and L > 1:
            K('lay_vmix', g.E, 1, (g.N, g.E, L, h, g.eI, g.eJ, self.vmix, dt, u, self.diss, self.vmix_cd))

    def energy(self, h, u):
        """Total energy per unit density, Boussinesq form (reference layers.py:234-253)."""
        gh = self.dg.host
        hh, uu, b = np.asarray(h), np.asarray(u), self.b
        ce = np.where(gh.cellEdge >= 0, gh.cellEdge, 0)
        ok = gh.cellEdge >= 0
        kin = sum(np.sum(hh[k] * np.sum(np.where(ok, gh.le[ce] * gh.de[ce] * 0.25 * uu[k][ce] ** 2, 0.0), axis=1)) for k in range(self.L))
        z = b + np.cumsum(hh[::-1], axis=0)[::-1]
        pot = np.sum(gh.areaCell * self.grav * (z[0] ** 2 - b ** 2) / 2)
        for k in range(1, self.L):
            pot += np.sum(gh.areaCell * self.gp[k - 1] * (z[k] ** 2 - b ** 2) / 2)
        return float(kin + pot)


class Transport:
    def __init__(self, dg, layers=1, beta=BETA, tracers=1, backend='oracle'):
        self.K = kernels(backend)
        self.dg, self.L, self.beta, self.T = dg, layers, beta, tracers
        N, E = dg.N, dg.E
        R = tracers * layers
        self.psi, self.td, self.p1, self.p2, self.Rp, self.Rm, self.out = (np.zeros((R, N)) for _ in range(7))
        self.Hf, self.A = np.zeros((R, E)), np.zeros((R, E))

    def mass_after(self, M0, Fm, M1):
        g = self.dg
        self.K('mass_update', g.N, self.L, (g.N, g.E, M0, Fm, g.cellEdgeAsc, g.eI, M1))

    def step(self, M0, M1, Fm, psi, order=3):
        return self.step_many(M0, M1, Fm, [psi], order)[0]

    def step_many(self, M0, M1, Fm, tracers, order=3):
        g, K = self.dg, self.K
        n, L, N, E = len(tracers), self.L, g.N, g.E
        assert n <= self.T
        R = n * L
        psi, td, p1, p2, Rp, Rm, out = (a[:R] for a in (self.psi, self.td, self.p1, self.p2, self.Rp, self.Rm, self.out))
        Hf, A = self.Hf[:R], self.A[:R]
        for j, t in enumerate(tracers):
            np.copyto(psi[j * L:(j + 1) * L], t)
        b = self.beta
        K('tr_td', N, R, (N, E, L, M0, psi, Fm, M1, g.cellEdgeAsc, g.eI, g.eJ, td))
        if order == 1:
            res = td
        else:
            for src, frac, dst in ((psi, 1 / 3, p1), (p1, 1 / 2, p2)):
                K('tr_hflux', E, R, (E, L, src, src, frac, Fm, g.d2idx, g.d2wt_tr, g.eI, g.eJ, N, b, Hf))
                K('tr_stage', N, R, (N, E, L, M0, psi, Hf, frac, Fm, g.cellEdgeAsc, g.eI, dst))
            K('tr_aflux', E, R, (E, L, psi, p2, p2, Fm, g.d2idx, g.d2wt_tr, g.eI, g.eJ, N, b, A))
            K('tr_ratios', N, R, (N, E, L, psi, td, M1, A, g.nbr, g.cellEdgeAsc, g.eI, Rp, Rm))
            K('tr_apply', N, R, (N, E, L, td, M1, A, Rp, Rm, g.cellEdgeAsc, g.eI, g.eJ, out))
            res = out
        for j, t in enumerate(tracers):
            np.copyto(t, res[j * L:(j + 1) * L])
        return tracers


def dsum(x, y=None, backend='oracle'):
    return kernels(backend).dsum(x, y)


def build(verbose=False):
    """Compile oracle.c into liboracle.so (gcc, no FMA contraction, OpenMP)."""
    import subprocess
    cmd = ['gcc', '-O2', '-ffp-contract=off', '-fno-fast-math', '-fopenmp', '-shared', '-fPIC', '-Wall', '-o',
           str(HERE / 'liboracle.so'), str(HERE / 'oracle.c')]
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)
