"""Stacked-layer shallow water with a split-explicit fast mode, on the isw CUDA core (reference src/insilica/layers.py).

``Layers`` keeps the reference's constructor and methods (``step``, ``substeps``, ``lap_max``, ``energy``) and argument
meanings; the arrays are the caller's device arrays (h (L, N), u (L, E), Fm (L, E), FP64), updated in place on the
current CUDA stream. Air layers (``air=dict(cp=, kappa=, rd=)``: h is mass per area, ``step`` and ``update_gfast`` take
the layers' potential temperature theta, updated in place by the interfacial stress's heating) run in the FP64 form.
The option branches of Boussinesq layers are built in the FP64 form: thin walls (``wall``), the shelf and its bed flags
(``shelf``, ``shelf_bed``), and the per-step fields the ocean and the tides set as attributes (``sig`` with ``zm``,
``tide``, ``cd_bot``, ``cbot``). Air layers, walls and the shelf asked of the mixed form step in the FP64 form (the
object's ``precision`` says which form it runs).
"""
import ctypes
import math
import weakref

import numpy as np
import torch

from . import _lib
from .gpu import as_device_grid, device_ptr, dsum, stream_of

LMAX = 8
FAST_COURANT = 0.5          # fast sub-step: tau sqrt(gH) / d_min <= this (reference layers.py:31)
DIV_DAMP = 0.1              # divergence damping of the fast mode (reference layers.py:32)
GRAV = 9.80616
P0 = 1.0e5                  # reference pressure of potential temperature, Pa (reference constants.py:14)
R_DRY, CP_DRY = 287.04, 1004.6   # the dry air's constants (reference constants.py:8-10)
KAPPA = R_DRY / CP_DRY


class Layers:
    def __init__(self, dg, layers=1, b=None, grav=GRAV, gprime=(), drag=0.0, stress=0.0, nu4=0.0, floor=1.0, rotation=1.0,
                 div_damp=DIV_DAMP, air=None, vmix=0.0, thin=2.0, wall=None, thin_wind=0.0, shelf=0.0, vmix_cd=0.0,
                 shelf_bed=False, batched=True, precision=None):
        """The reference's constructor (layers.py:36-37). batched (this core's): FP64 Boussinesq layers without option
        branches step through a private one-stack batch (tiled fast loop, one graph; bit-identical results); False keeps
        the per-call kernels. precision (this core's): 'double' or 'mixed' for this object; None takes the grid's form
        (the precision switch in force when the DeviceGrid was made)."""
        if precision not in (None, 'double', 'mixed'):
            raise ValueError(f'Layers: precision {precision!r}, want double or mixed')
        dg = as_device_grid(dg)         # the reference's own DeviceGrid is accepted too (its host Grid is used)
        mixed = dg.mixed if precision is None else precision == 'mixed'
        if mixed and (air or wall is not None or shelf or shelf_bed):
            # air layers, walls and the shelf step in the FP64 form on a grid of either form (the reference's mixed
            # build keeps its air kernels in FP64 too); this object reports precision ISW_FP64
            mixed = False
        assert wall is None or not air, 'walls are for Boussinesq layers'
        assert 1 <= layers <= LMAX and len(gprime) == layers - 1
        self.dg, self.L = dg, layers
        self.grav, self.nu4, self.floor, self.div_damp, self.thin = grav, nu4, floor, div_damp, thin
        self.vmix, self.vmix_cd = vmix, vmix_cd
        self.thin_wind = thin_wind
        self.air = air
        # the air's constants (reference layers.py:64-65: cp 1004.6, kappa, R 287.04 unless the air dict gives them)
        self.cpa, self.kap, self.rda = (air or {}).get('cp', CP_DRY), (air or {}).get('kappa', KAPPA), (air or {}).get('rd', R_DRY)
        self.shelf = float(shelf)
        self._wall = None if wall is None else np.ascontiguousarray(np.asarray(
            wall.detach().cpu().numpy() if isinstance(wall, torch.Tensor) else wall, dtype=np.float64).reshape(-1))
        self.wall = None if wall is None else torch.as_tensor(self._wall, device=f'cuda:{dg.device}')
        self._opts = dict(sig=None, tide=None, cbot=None, cd_bot=0.0)
        self._zm = None
        self.precision = _lib.ISW_MIXED if mixed else _lib.ISW_FP64
        self._b_host = np.zeros(dg.N) if b is None else np.ascontiguousarray(np.asarray(
            b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else b, dtype=np.float64))
        self.b = torch.as_tensor(self._b_host, device=f'cuda:{dg.device}')
        gp = np.ascontiguousarray(np.asarray(gprime, dtype=np.float64).reshape(-1)) if layers > 1 else np.zeros(1)
        self._drag = np.ascontiguousarray(np.broadcast_to(np.asarray(drag, dtype=np.float64), (layers,)))
        self._stress = np.ascontiguousarray(np.broadcast_to(np.asarray(stress, dtype=np.float64), (layers,)))
        self.gp = gp
        p = _lib.LayersParams(L=layers, grav=float(grav), gprime=_lib.host_ptr(gp), drag=_lib.host_ptr(self._drag),
                              stress=_lib.host_ptr(self._stress), nu4=float(nu4), floor_=float(floor), rotation=float(rotation),
                              div_damp=float(div_damp), thin=float(thin), vmix=float(vmix), vmix_cd=float(vmix_cd),
                              b=_lib.host_ptr(self._b_host), precision=self.precision, air=1 if air else 0,
                              cp=float(self.cpa), kappa=float(self.kap), rd=float(self.rda), p0=P0,
                              thin_wind=float(thin_wind), wall=_lib.host_ptr(self._wall) if self._wall is not None else None,
                              shelf=float(shelf), shelf_bed=1 if shelf_bed else 0, percall=0 if batched else 1)
        h = ctypes.c_void_p()
        _lib.check(_lib.isw_layers_create(dg.handle, ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.dmin = float(np.min(dg.host.de))
        self._L1 = None
        self.k = KernelTable(self)

    def __del__(self):
        h = getattr(self, '_h', None)
        destroy = getattr(_lib, 'isw_layers_destroy', None) if _lib is not None else None
        if h is not None and h.value and destroy is not None:      # (module globals are gone at interpreter exit)
            destroy(h)
            self._h = None

    # the per-step fields of the option branches, set as attributes as the reference's callers do (ocean.py:159,
    # tides.py:64-69); the arrays are borrowed by the core until replaced or set to None
    def _set(self, name, code, a, shape, value=0.0):
        ptr = None if a is None else device_ptr(a, shape=shape, name=name, device=self.dg.device)
        _lib.check(_lib.isw_layers_set_option(self._h, code, ptr, float(value)))
        self._opts[name] = a

    @property
    def sig(self):
        return self._opts['sig']

    @sig.setter
    def sig(self, a):
        self._set('sig', _lib.ISW_OPT_SIG, a, (self.L, self.dg.N))

    @property
    def zm(self):
        """The layers' mid-heights of the per-cell buoyancy form; the core keeps its own (an assigned array is unused)."""
        return self._zm

    @zm.setter
    def zm(self, a):
        self._zm = a

    @property
    def tide(self):
        return self._opts['tide']

    @tide.setter
    def tide(self, a):
        self._set('tide', _lib.ISW_OPT_TIDE, a, (self.dg.N,))

    @property
    def cbot(self):
        return self._opts['cbot']

    @cbot.setter
    def cbot(self, a):
        self._set('cbot', _lib.ISW_OPT_CBOT, a, (self.dg.E,))

    @property
    def cd_bot(self):
        return self._opts['cd_bot']

    @cd_bot.setter
    def cd_bot(self, v):
        _lib.check(_lib.isw_layers_set_option(self._h, _lib.ISW_OPT_CD_BOT, None, float(v)))
        self._opts['cd_bot'] = float(v)

    def _shapes(self):
        return (self.L, self.dg.N), (self.L, self.dg.E)

    def mask(self, a, rows, stream=None):
        """Zero the wall edges of the first `rows` rows of the edge field a (rows, E) in place; a no-op without walls
        (reference layers.py:94-97)."""
        if self._wall is None:
            return
        dev = self.dg.device
        _lib.check(_lib.isw_layers_mask(self._h, device_ptr(a, name='a', device=dev, numel=int(rows) * self.dg.E), int(rows),
                                        stream_of(dev, stream)))

    def set_bottom(self, b, stream=None):
        """Replace the bottom height the layers rest on (N values): the core's copy and this object's `b`."""
        bt = b if isinstance(b, torch.Tensor) else torch.as_tensor(np.asarray(b, dtype=np.float64))
        bt = bt.to(device=self.b.device, dtype=torch.float64).contiguous()
        _lib.check(_lib.isw_layers_set_bottom(self._h, device_ptr(bt, shape=(self.dg.N,), name='b', device=self.dg.device),
                                              stream_of(self.dg.device, stream)))
        self.b.copy_(bt)

    def status(self, reset=False, stream=None):
        """The status word of the one-stack batch this Layers steps through: 0, ISW_ETIMEOUT (5) after a fast-loop barrier
        timed out, or ISW_ENOTFINITE (6) after a step left a NaN or Inf thickness. While it is set, step() raises; reset
        clears it (restore the state first)."""
        st = _lib.isw_layers_status(self._h, stream_of(self.dg.device, stream), 1 if reset else 0)
        if st not in (_lib.ISW_OK, _lib.ISW_ETIMEOUT, _lib.ISW_ENOTFINITE):
            _lib.check(st)
        return st

    def step(self, h, u, dt, nfast, Fm=None, theta=None, stream=None):
        """One time-split RK3 step in place on h (L, N), u (L, E), with nfast fast sub-steps per full step (stage s takes
        ceil(c_s nfast)). Fm, if given, receives each layer's final-stage volume flux l dt F (m^3; for air layers the
        mass flux, kg). Air layers take theta (L, N), which the interfacial stress's heating updates in place."""
        sh, su = self._shapes()
        dev = self.dg.device
        if bool(self.air) != (theta is not None):
            raise ValueError('Layers.step: theta is required for air layers and only for them')
        if self.nu4:
            self.nu4dt = self.nu4 * dt             # the step's nabla^4 loss, booked as heat by an air exchange (layers.py:202)
        ph = device_ptr(h, shape=sh, name='h', device=dev)
        pu = device_ptr(u, shape=su, name='u', device=dev)
        pf = device_ptr(Fm, shape=su, name='Fm', device=dev)
        if self.air:
            pt = device_ptr(theta, shape=sh, name='theta', device=dev)
            _lib.check(_lib.isw_layers_step_air(self._h, ph, pu, pf, pt, float(dt), int(nfast), stream_of(dev, stream)))
            return
        _lib.check(_lib.isw_layers_step(self._h, ph, pu, pf, float(dt), int(nfast), stream_of(dev, stream)))

    def substeps(self, h, dt, stream=None):
        """Fast sub-steps per full step for the current deepest column (reference layers.py:99-102)."""
        sh, _ = self._shapes()
        out = ctypes.c_int()
        _lib.check(_lib.isw_layers_substeps(self._h, device_ptr(h, shape=sh, name='h', device=self.dg.device), float(dt),
                                            ctypes.byref(out), stream_of(self.dg.device, stream)))
        return out.value

    def lap(self, u, out, stream=None):
        """out = the edge vector Laplacian of u (reference layers.py:123-127)."""
        _, su = self._shapes()
        dev = self.dg.device
        _lib.check(_lib.isw_layers_lap(self._h, device_ptr(u, shape=su, name='u', device=dev),
                                       device_ptr(out, shape=su, name='out', device=dev), stream_of(dev, stream)))

    def lap_max(self, iters=30):
        """Largest |eigenvalue| of the edge vector Laplacian by power iteration from a fixed seed, 1/m^2
        (reference layers.py:111-121). Norms are deterministic tree sums."""
        dev = f'cuda:{self.dg.device}'
        v = torch.as_tensor(np.random.default_rng(0).standard_normal((self.L, self.dg.E)), device=dev)
        out = torch.empty_like(v)
        lam = 0.0
        for _ in range(iters):
            self.lap(v, out)
            n1 = math.sqrt(dsum(out[0], out[0]))
            lam = n1 / math.sqrt(dsum(v[0], v[0]))
            v = out / n1
            out = torch.empty_like(v)
        return lam

    def update_gfast(self, h, theta, stream=None):
        """Air layers: each cell's fast-mode coefficient R T_s / mu (+ its interfaces' terms) from the current state
        (reference layers.py:104-109); substeps() then uses it. A no-op for Boussinesq layers."""
        if self.air:
            sh, _ = self._shapes()
            dev = self.dg.device
            _lib.check(_lib.isw_layers_update_gfast(self._h, device_ptr(h, shape=sh, name='h', device=dev),
                                                    device_ptr(theta, shape=sh, name='theta', device=dev), stream_of(dev, stream)))

    def exchange(self, wx, h, u, M, psi, theta=None, seq=False, stream=None):
        """Move thickness wx (L-1, N; positive upward across the interface below layer k) between layers with its tracer
        psi and momentum, conservatively (reference layers.py:214-232); M (L, N) the layers' mass. For air layers with
        theta given, the kinetic energy the momentum mixing removed (and the last step's nabla^4 loss) warms the column
        and a nearly empty layer takes its neighbours' wind (thin_wind). seq: the tracer moves in the order water passes
        through the column. The caller keeps donors above the floor."""
        sh, su = self._shapes()
        dev = self.dg.device
        if self.L < 2:
            return
        pt = device_ptr(theta, shape=sh, name='theta', device=dev) if theta is not None else None
        _lib.check(_lib.isw_layers_exchange(self._h, device_ptr(wx, shape=(self.L - 1, self.dg.N), name='wx', device=dev),
                                            device_ptr(h, shape=sh, name='h', device=dev), device_ptr(u, shape=su, name='u', device=dev),
                                            device_ptr(M, shape=sh, name='M', device=dev), device_ptr(psi, shape=sh, name='psi', device=dev),
                                            pt, 1 if seq else 0, stream_of(dev, stream)))

    def energy(self, h, u, theta=None):
        """Total energy per unit density (J/rho0; reference layers.py:234-253), on the host. Air layers: kinetic plus
        enthalpy sum mu pibar theta plus the ground's potential g b mu."""
        gh = self.dg.host
        hh = h.detach().cpu().numpy() if isinstance(h, torch.Tensor) else np.asarray(h)
        uu = u.detach().cpu().numpy() if isinstance(u, torch.Tensor) else np.asarray(u)
        b = self._b_host
        ce = np.where(gh.cellEdge >= 0, gh.cellEdge, 0)
        ok = gh.cellEdge >= 0
        kin = sum(np.sum(hh[k] * np.sum(np.where(ok, gh.le[ce] * gh.de[ce] * 0.25 * uu[k][ce] ** 2, 0.0), axis=1)) for k in range(self.L))
        if self.air:
            if theta is None:
                raise ValueError('Layers.energy: air layers need theta')
            th = theta.detach().cpu().numpy() if isinstance(theta, torch.Tensor) else np.asarray(theta)
            p = np.cumsum(self.grav * hh, axis=0)
            pt = np.vstack([np.zeros((1, hh.shape[1])), p[:-1]])
            pib = self.cpa * (p ** (self.kap + 1) - pt ** (self.kap + 1)) / ((self.kap + 1) * (p - pt) * P0 ** self.kap)
            return float(kin + np.sum(gh.areaCell * (np.sum(hh * pib * th, axis=0) + self.grav * b * hh.sum(0))))
        z = b + np.cumsum(hh[::-1], axis=0)[::-1]
        pot = np.sum(gh.areaCell * self.grav * (z[0] ** 2 - b ** 2) / 2)
        for k in range(1, self.L):
            pot += np.sum(gh.areaCell * self.gp[k - 1] * (z[k] ** 2 - b ** 2) / 2)
        return float(kin + pot)


def _numel(a):
    if isinstance(a, torch.Tensor):
        return a.numel()
    if hasattr(a, '__cuda_array_interface__'):
        return int(np.prod(a.__cuda_array_interface__['shape'], dtype=np.int64))
    return torch.from_dlpack(a).numel()


class KernelTable:
    """The entries of the reference's kernel table (``Layers.k``, layers.py:83-91) that its callers launch themselves,
    with the reference's launch convention ``k[name](grid, block, args)``: ``'vmix_heat'`` (world.py:317-318, after the
    sea coupling) and ``'lay_mask'``. The grid and block sizes are the caller's CuPy launch shape and are not needed: each
    entry runs this core's kernel for the whole field. The arguments are read in the reference kernels' order, with
    their device arrays' sizes checked; the grid tables passed must be this Layers' grid's."""

    def __init__(self, core):
        self._ref = weakref.ref(core)        # no reference cycle: a Layers is freed as soon as its last user lets go

    @property
    def _core(self):
        c = self._ref()
        if c is None:
            raise RuntimeError('Layers.k: the Layers object is gone')
        return c

    def __contains__(self, name):
        return name in ('vmix_heat', 'lay_mask')

    def __getitem__(self, name):
        if name == 'vmix_heat':
            return self._vmix_heat
        if name == 'lay_mask':
            return self._lay_mask
        raise KeyError(f'Layers.k[{name!r}]: only vmix_heat and lay_mask are launched by callers; the other kernels run '
                       'inside this core\'s step')

    def _vmix_heat(self, grid, block, args, stream=None, **kw):
        """args = (N, L, h, diss, cellEdge, le, de, areaCell, grav, cp, kappa, p0, theta), the reference kernel's order."""
        c = self._core
        N, L, h, diss, cellEdge, le, de, areaCell, grav, cpa, kap, p0, theta = args
        if int(N) != c.dg.N or int(L) != c.L:
            raise ValueError(f'vmix_heat: N {int(N)}, L {int(L)}; this Layers has N {c.dg.N}, L {c.L}')
        for nm, a, n in (('cellEdge', cellEdge, 6 * c.dg.N), ('le', le, c.dg.E), ('de', de, c.dg.E), ('areaCell', areaCell, c.dg.N)):
            if _numel(a) != n:
                raise ValueError(f'vmix_heat: {nm} has {_numel(a)} values, the grid {n}')
        dev = c.dg.device
        sh = (c.L, c.dg.N)
        _lib.check(_lib.isw_layers_vmix_heat(c._h, device_ptr(h, shape=sh, name='h', device=dev),
                                             device_ptr(diss, name='diss', device=dev, numel=c.dg.E),
                                             device_ptr(theta, shape=sh, name='theta', device=dev), float(grav), float(cpa),
                                             float(kap), float(p0), stream_of(dev, stream)))

    def _lay_mask(self, grid, block, args, stream=None, **kw):
        """args = (E, rows, wall, a), the reference kernel's order; the wall is this Layers' own."""
        c = self._core
        E, rows, wall, a = args
        if int(E) != c.dg.E:
            raise ValueError(f'lay_mask: E {int(E)}, the grid {c.dg.E}')
        c.mask(a, int(rows), stream=stream)

