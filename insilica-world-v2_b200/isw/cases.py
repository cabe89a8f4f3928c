"""Initial states for the dynamical core's workloads (host NumPy, set-up only).

Single-layer benchmarks restate the reference's analytic cases (reference ``src/insilica/cases.py``):
Williamson 2 (``cases.py:49-53``), the Galewsky jet (``cases.py:73-95``), the cosine bell (``cases.py:32-35``) and
the default step (``cases.py:38-40``); the hyperviscosity rule restates ``world.py:48-52``.

The stacked-layer workloads (``stack_state``) are this project's own seeded synthetic states: L Boussinesq layers with
balanced zonal jets (the L-layer form of ``cases.py:152-171``), random spherical-harmonic topography, a smooth 1%
random thickness perturbation, and FCT tracers (potential temperature, vapour, a gas tracer).
"""
import math

import numpy as np

R_PLANET = 6.371e6
OMEGA_REF = 2 * math.pi / 86400          # the reference's rotation (reference constants.py:5)
OMEGA_EARTH = 7.292e-5                    # the sidereal rotation the stacked workloads use
GRAV = 9.80616


def planet_of(g):
    return getattr(g, 'radius', R_PLANET), getattr(g, 'omega', OMEGA_REF), getattr(g, 'grav', GRAV)


def edge_east_north(g):
    """Latitude, longitude and east/north components of each edge normal at the Voronoi edge midpoint xm
    (reference cases.py:16-25)."""
    x = g.xm
    lat = np.arcsin(np.clip(x[:, 2], -1, 1))
    lon = np.arctan2(x[:, 1], x[:, 0])
    en = -np.sin(lon) * g.ne[:, 0] + np.cos(lon) * g.ne[:, 1]
    nn = (-np.sin(lat) * np.cos(lon) * g.ne[:, 0] - np.sin(lat) * np.sin(lon) * g.ne[:, 1] + np.cos(lat) * g.ne[:, 2])
    return lat, lon, en, nn


def great_circle(g, lon_c, lat_c):
    c = np.array([math.cos(lat_c) * math.cos(lon_c), math.cos(lat_c) * math.sin(lon_c), math.sin(lat_c)])
    return R_PLANET * np.arccos(np.clip(g.pos @ c, -1, 1))


def cosine_bell(g, lon_c=3 * math.pi / 2, lat_c=0.0, radius=R_PLANET / 3, height=1000.0):
    """Williamson 1's cosine bell (reference cases.py:32-35)."""
    dist = great_circle(g, lon_c, lat_c)
    return np.where(dist < radius, 0.5 * height * (1 + np.cos(math.pi * dist / radius)), 0.0)


def default_dt(n):
    """450 s at n = 4, halved per level (reference cases.py:38-40)."""
    return 450.0 * 2.0 ** (4 - n)


def visc4(g, U):
    """nu4 = U d^3 / pi^4 with d the mean edge spacing (reference world.py:48-52)."""
    d = float(np.mean(g.de))
    return U * d ** 3 / math.pi ** 4


def solid_body_flux(g, dt, alpha=math.pi / 2 - 0.05, period_days=12):
    """Solid-body rotation's edge normal winds (reference tests/test_accuracy.py:25-29) and the volume flux per step
    l u dt, for transport-only runs."""
    u0 = 2 * math.pi * R_PLANET / (period_days * 86400)
    om = np.array([-math.sin(alpha) * u0 / R_PLANET, 0, math.cos(alpha) * u0 / R_PLANET])
    un = np.sum(np.cross(om, g.xm * R_PLANET) * g.ne, axis=1)
    return un, un * g.le * dt


def _galewsky_u(phi, umax=80.0, p0=math.pi / 7):
    p1 = math.pi / 2 - p0
    e_n = math.exp(-4 / (p1 - p0) ** 2)
    phi = np.asarray(phi, dtype=float)
    inside = (phi > p0) & (phi < p1)
    with np.errstate(divide='ignore', over='ignore', invalid='ignore'):
        v = umax / e_n * np.exp(1 / ((phi - p0) * (phi - p1)))
    return np.where(inside, v, 0.0)


def _gradient_wind(ujet, a, Om, M=20000):
    """dM/dphi = -a u (f + u tan(phi) / a) integrated from the south pole on M midpoint cells; returns (ph, M(phi))."""
    dphi = math.pi / M
    ph = -math.pi / 2 + (np.arange(1, M + 1) - 0.5) * dphi
    uu = ujet(ph)
    return dphi, np.concatenate([[0.0], np.cumsum(-a * uu * (2 * Om * np.sin(ph) + np.tan(ph) * uu / a) * dphi)])


def _interp(g_lat, dphi, Mv, M=20000):
    x = (g_lat + math.pi / 2) / dphi
    k = np.minimum(M - 1, np.floor(x).astype(int))
    return Mv[k] + (x - k) * (Mv[k + 1] - Mv[k])


def initial_state(g, preset):
    """One layer (h, b, u) for 'w2' or 'galewsky' (reference cases.py:43-98)."""
    a, Om, G = planet_of(g)
    lat_e, lon_e, en, nn = edge_east_north(g)
    b = np.zeros(g.N)
    if preset == 'w2':
        u0, gh0 = 2 * math.pi * a / (12 * 86400), 2.94e4
        s = np.sin(g.lat)
        h = (gh0 - (a * Om * u0 + u0 * u0 / 2) * s * s) / G
        u = u0 * np.cos(lat_e) * en
    elif preset == 'galewsky':
        dphi, gh = _gradient_wind(_galewsky_u, a, Om)
        h = _interp(g.lat, dphi, gh) / G
        h = h + 10000 - np.sum(h * g.areaCell) / np.sum(g.areaCell)
        h = h + 120 * np.cos(g.lat) * np.exp(-((g.lon / (1 / 3)) ** 2)) * np.exp(-(((math.pi / 4 - g.lat) / (1 / 15)) ** 2))
        u = _galewsky_u(lat_e) * en
    else:
        raise ValueError(f'unknown single-layer case {preset!r}')
    return h, b, u


# ---- random fields on the sphere ----

def sh_field(g, rng, lmax, spectrum, device=None):
    """A real random spherical-harmonic field at the cells: sum over l <= lmax, m <= l of 4pi-normalised associated
    Legendre functions times N(0, spectrum(l) / (2l + 1)) coefficients on cos(m lon) and sin(m lon); area-weighted
    RMS normalised to 1. device: evaluate the sum with torch on that CUDA device (the same coefficients, drawn in the same
    order; the sum rounds differently), for the many members of ensembles and serving runs."""
    if device is not None:
        import torch
        xp = torch
        T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
        lat, lon = T(g.lat), T(g.lon)
    else:
        xp = np
        lat, lon = g.lat, g.lon
    x = xp.sin(lat)
    c = xp.sqrt(xp.clamp(1 - x * x, min=0.0) if xp is not np else np.maximum(0.0, 1 - x * x))
    f = xp.zeros_like(x)
    pmm = xp.ones_like(x)
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * c * math.sqrt((2 * m + 1) / (2 * m)) * (math.sqrt(2.0) if m == 1 else 1.0)
        cm, sm = xp.cos(m * lon), xp.sin(m * lon)
        p2, p1 = None, pmm
        for l in range(m, lmax + 1):
            if l == m:
                p = pmm
            elif l == m + 1:
                p = math.sqrt(2 * m + 3) * x * pmm
            else:
                A = math.sqrt((4 * l * l - 1) / (l * l - m * m))
                B = math.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
                p = A * (x * p1 - B * p2)
            if l > m:
                p2, p1 = p1, p
            if l == 0:
                continue
            s = math.sqrt(spectrum(l) / (2 * l + 1))
            a = rng.standard_normal() * s
            if m > 0:
                f += p * (a * cm + (rng.standard_normal() * s) * sm)
            else:
                f += p * (a * cm)
    if device is not None:
        f = f.cpu().numpy()
    A = g.areaCell / np.sum(g.areaCell)
    f = f - np.sum(A * f)
    return f / math.sqrt(np.sum(A * f * f))


def topography(g, seed, lmax=32, rms=2000.0, device=None):
    """Random spherical-harmonic topography to degree lmax with the given area-weighted RMS (m), flat spectrum."""
    return rms * sh_field(g, np.random.default_rng(seed), lmax, lambda l: 1.0, device)


def smooth_noise(g, seed, corr=1.0e6, lmax=48, device=None):
    """Unit-RMS smooth random field with a Gaussian correlation of length corr (m)."""
    k = (corr / R_PLANET) ** 2 / 2
    return sh_field(g, np.random.default_rng(seed), lmax, lambda l: math.exp(-k * l * (l + 1)), device)


# ---- stacked-layer workloads ----

def jet_profile(U, lat0=math.radians(45.0), width=math.radians(10.0)):
    return lambda phi: U * np.exp(-((np.asarray(phi, dtype=float) - lat0) / width) ** 2)


def balanced_layers(g, H, ujets, gprime, b, floor, omega, grav=GRAV, M=20000):
    """L Boussinesq layers (top first) with zonal winds ujets[k](phi), each in gradient-wind balance:
    M_0 = g eta, M_k = M_{k-1} + g'_{k-1} z_k (z_k the top of layer k), the L-layer form of reference
    cases.py:152-171. Interface area means sit at mean(b) + sum of the thicknesses below; the stack rests on b,
    with every layer at least `floor` thick where the terrain rises through it."""
    a = R_PLANET
    L = len(H)
    Ms = []
    for uj in ujets:
        dphi, Mv = _gradient_wind(uj, a, omega, M)
        Ms.append(_interp(g.lat, dphi, Mv, M))
    A = g.areaCell / np.sum(g.areaCell)
    bm = float(np.sum(A * b))
    z = []
    for k in range(L):
        zv = Ms[0] / grav if k == 0 else (Ms[k] - Ms[k - 1]) / gprime[k - 1]
        z.append(zv + bm + sum(H[k:]) - np.sum(A * zv))
    h = np.zeros((L, g.N))
    s = b.copy()
    for k in range(L - 1, -1, -1):
        h[k] = np.maximum(z[k] - s, floor)
        s = s + h[k]
    lat_e, _, en, _ = edge_east_north(g)
    u = np.stack([uj(lat_e) * en for uj in ujets])
    return h, u


STACKS = {
    # three Boussinesq air layers of 2.5 / 3.5 / 4 km with jets 30 / 25 / 20 m/s at 45N. g' 2 and 1 m/s^2 keep the
    # grid-scale internal wave inside RK3's stability range at the stacks' step (stack_dt). The interfacial stress
    # (5e-4 m/s: a 40-day decay between km-thick layers) locks a layer pressed to its floor over a peak to its neighbour;
    # its quadratic part (cd 1e-3, the reference's Earth-preset interface drag) stops the wind of a layer squeezed to its
    # floor at a front from running away (without it some seeds blow up within days at levels 6 and 7)
    'air': dict(H=(2500.0, 3500.0, 4000.0), U=(30.0, 25.0, 20.0), gprime=(2.0, 1.0), base=0.0, floor=1.0,
                stress=(0.0, 0.0, 0.0), visc4_U=20.0, knee=800.0, cap=1500.0, vmix=5e-4, vmix_cd=1e-3),
    # two ocean layers of 100 / 3900 m over a flat 4 km basin floor; one barotropic 20 m/s jet (the lower layer's scaled
    # by 1 + g'/g so the interface stays parallel to the surface); bottom stress, and the reference ocean's interfacial
    # stress (its interface_stress 5e-4, reference ocean.py:32), which keeps a top layer thinned to its floor locked to the
    # layer below instead of running away. The terrain stays under the air stack only: a 20 m/s barotropic jet over
    # 2 km of random relief outruns the step within a day.
    'ocean': dict(H=(100.0, 3900.0), U=(20.0, 20.0 * (1 + 0.016 / GRAV)), gprime=(0.016,), base=-4000.0, floor=1.0,
                  stress=(0.0, 2.5e-4), visc4_U=0.5, vmix=5e-4, vmix_cd=1e-3, flat=True),
}


def stack_dt(n):
    """The stacked workloads' step: 300 s at n = 6, doubling per coarser level; 120 s at n = 7. The grid-scale internal
    wave carried by the 30 m/s jet, (c1 + U) k_max dt with c1 = 64 m/s and k_max^2 the vector Laplacian's largest
    eigenvalue, then stays near 1.2 through level 6, inside RK3's sqrt(3); at level 7 the resolved fronts carry faster
    winds (50-80 m/s), and 150 s let some seeds' air stacks blow up within days where 120 s holds them 30 days."""
    return 120.0 * 2.0 ** (7 - n) if n >= 7 else 1200.0 * 2.0 ** (4 - n)


def compress_peaks(t, knee, cap):
    """Terrain t unchanged below knee, compressed smoothly toward cap above it (tanh), so no peak pierces the
    stack's lowest interface: a Boussinesq layer pressed to its floor against a slope feels g' grad(b) with nothing to
    balance it (the reference treats that case with its shelf option, which these workloads leave off)."""
    w = cap - knee
    return np.where(t <= knee, t, knee + w * np.tanh((t - knee) / w))


def stack_state(g, kind, seed, perturb=0.01, ntracers=3, topo=None, omega=OMEGA_EARTH, device=None):
    """A stacked-layer workload: dict(h (L, N), u (L, E), b (N), gprime, stress, nu4, floor, tracers [T x (L, N)]).
    Topography: random spherical harmonics to degree 32, 2 km RMS (seeded, shared by the stacks of one seed), its peaks
    above 800 m compressed toward 1.5 km, under the air stack; the ocean stack lies on a flat 4 km floor. Each layer's thickness is scaled by
    (1 + perturb r_k), r_k a unit-RMS random field with a 1000 km correlation length. Tracers (per cell and layer,
    i.i.d.): potential temperature U(250, 310) K, vapour log-normal (median 5e-3, sigma_ln 0.5), a gas U(0, 1).
    device: synthesise the random fields on that CUDA device (faster; equal to the host's to rounding)."""
    c = STACKS[kind]
    L = len(c['H'])
    if c.get('flat'):
        b = np.full(g.N, c['base'])
    else:
        t = topography(g, seed, device=device) if topo is None else topo
        b = c['base'] + compress_peaks(t, c['knee'], c['cap'])
    ujets = [jet_profile(U) for U in c['U']]
    h, u = balanced_layers(g, c['H'], ujets, c['gprime'], b, c['floor'], omega)
    for k in range(L):
        h[k] = np.maximum(h[k] * (1 + perturb * smooth_noise(g, seed * 100 + 10 + k, device=device)), c['floor'])
    rng = np.random.default_rng(seed * 100 + 50)
    tr = [rng.uniform(250.0, 310.0, (L, g.N)), 5e-3 * np.exp(0.5 * rng.standard_normal((L, g.N))),
          rng.uniform(0.0, 1.0, (L, g.N))][:ntracers]
    return dict(h=h, u=u, b=b, gprime=list(c['gprime']), stress=list(c['stress']), floor=c['floor'],
                nu4=visc4(g, c['visc4_U']), vmix=c.get('vmix', 0.0), vmix_cd=c.get('vmix_cd', 0.0), tracers=tr, L=L, kind=kind)
