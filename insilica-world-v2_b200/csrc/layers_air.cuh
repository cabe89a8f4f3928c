// Phase functions of the air branch of the time-split RK3 step, plain FP64 form (reference layers.py:104-109, 134-136,
// 152-166, 187-192, 203-206; kernels/layers.cu:110-250, 596-621). Air layers carry h = mass per area (kg/m^2) and a
// potential temperature theta per layer; hydrostatics from p = 0 at the top, Exner pi(p) = cp (p / p0)^kappa.
//   step start  cells: the column stiffness S (air_stiff, layers.cu:163-176)
//   stage A     cells: Montgomery potential with kinetic energy B and the layers' mass-mean Exner pibar (air_bern,
//               layers.cu:118-155); the PV pass is the Boussinesq one
//   stage E     edges: the Boussinesq pass, and the fast state uf = u0, accL = 0 (layers.py:154-156); cells: muf = h0
//   stage S     the Boussinesq slow tendency plus pibar grad(theta) (lay_slow's air term, layers.cu:322-326)
//   fast loop   cells: every layer's mass step and the forward-weighted linear potential phi (af_muphi, :189-213);
//               edges: every layer's wind (af_u, :215-223)
//   stage C     the layer fluxes hedge accL / n (af_flux, :226-230), recomputed per cell edge with the eI cell storing
//               them, and the floor limiter's scale (lay_scale)
//   stage D     h with the limited fluxes (lay_h); u = uf and Fm (lay_limit)
//   after       interfacial stress (Boussinesq vmix_edge) and its heat returned to theta (vmix_heat, :604-621)
//   any time    the fast mode's coefficient per cell Gc = R T_s / mu + interface terms (air_gfast, :239-252)
// Each function restates the reference kernel's arithmetic in its operation order (compiled with -fmad=false); pow
// comes from CUDA's libm, whose last bit may differ from the host's, so results hold to 1e-12 of the reference's.
#pragma once
#include "common.cuh"
#include "layers_fp64.cuh"

namespace isw {
namespace fp64 {

// one pow per interface: x_k = (p_k / p0)^kappa at the bottom of layer k
template <int L>
__device__ __forceinline__ void air_stiff_cell(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ theta,
                                               int i) {
  const int N = M.g.N;
  double p = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    p += M.grav * h[(size_t)k * N + i];
    const double dth = theta[(size_t)k * N + i] - (k + 1 < L ? theta[(size_t)(k + 1) * N + i] : 0.0);
    const double dpi = M.kap * M.cpa * pow(p / M.p0, M.kap) / p;
    M.S[(size_t)k * N + i] = dth > 0 ? dth * M.grav * dpi : 0.0;
  }
}

// Stage A for air, cells: the layers' mass-mean Exner function pibar (from the pressures at each layer's top and
// bottom), the Montgomery potential summed up from the ground with each interface's theta jump, the stiffness potential
// summed down from the top with the mass above, and the kinetic energy of the cell's edges.
template <int L>
__device__ __forceinline__ void air_bern_cell(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u,
                                              const double *__restrict__ theta, int i) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  double exner_bot[L];                       // (p / p0)^kappa at each layer's bottom
  double pbot = 0, exner_top = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double mass = h[(size_t)k * N + i];
    const double ptop = pbot;
    pbot = pbot + M.grav * mass;
    const double xk = pow(pbot / M.p0, M.kap);
    exner_bot[k] = xk;
    M.pibar[(size_t)k * N + i] = M.cpa * (pbot * xk - ptop * exner_top) / ((M.kap + 1) * (pbot - ptop));
    exner_top = xk;
  }
  double mont = M.grav * M.b[i] + theta[(size_t)(L - 1) * N + i] * M.cpa * exner_bot[L - 1];
  double mont_k[L];
  mont_k[L - 1] = mont;
#pragma unroll
  for (int k = L - 2; k >= 0; k--) {
    mont = mont + (theta[(size_t)k * N + i] - theta[(size_t)(k + 1) * N + i]) * M.cpa * exner_bot[k];
    mont_k[k] = mont;
  }
  double load[L], stiff_pot[L];             // mass down to each layer's bottom; the stiffness potential below
  double above = 0;
#pragma unroll
  for (int k = 0; k < L; k++) { above += h[(size_t)k * N + i]; load[k] = above; }
  double pot = 0;
#pragma unroll
  for (int k = L - 1; k >= 0; k--) { pot += M.S[(size_t)k * N + i] * load[k]; stiff_pot[k] = pot; }
  int es[6];
  double kin[6];                             // l_e d_e / 4 of each slot
  slots6(g.cellEdge, i, es);
#pragma unroll
  for (int t = 0; t < 6; t++) {
    const int e = es[t];
    kin[t] = e >= 0 ? g.le[e] * g.de[e] * 0.25 : 0.0;
  }
  const double area = g.areaCell[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *ul = u + (size_t)k * E;
    double ke = 0;
#pragma unroll
    for (int t = 0; t < 6; t++)
      if (es[t] >= 0) {
        const double ue = ul[es[t]];
        ke += kin[t] * ue * ue;
      }
    M.B[(size_t)k * N + i] = mont_k[k] - stiff_pot[k] + ke / area;
  }
}

// the stage's fast state: every layer's mass from h0 (cells) ...
template <int L>
__device__ __forceinline__ void air_fast_init_cell(const LayersDev &M, const double *__restrict__ h0, int i) {
  const int N = M.g.N;
#pragma unroll
  for (int k = 0; k < L; k++) M.muf[(size_t)k * N + i] = h0[(size_t)k * N + i];
}

// ... and every layer's wind from u0 with a zero sum (edges)
template <int L>
__device__ __forceinline__ void air_fast_init_edge(const LayersDev &M, const double *__restrict__ u0, int e) {
  const int E = M.g.E;
#pragma unroll
  for (int k = 0; k < L; k++) {
    M.uf[(size_t)k * E + e] = u0[(size_t)k * E + e];
    M.accL[(size_t)k * E + e] = 0.0;
  }
}

// A fast sub-step, cells: every layer's mass moved by its sub-step flux, then the forward-weighted fast potential
// summed down from the top: the stiffness times the damped mass load above each layer's bottom.
template <int L>
__device__ __forceinline__ void af_muphi_cell(const LayersDev &M, double tau, int i) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  int es[6];
  double flux_coef[6];                       // sign l_e of each slot
  slots6(g.cellEdge, i, es);
  int sg[6];
  signs6(g.cellSign, i, sg);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    flux_coef[s] = e >= 0 ? (double)sg[s] * g.le[e] : 0.0;
  }
  const double area = g.areaCell[i];
  double fast_load[L];
  double above = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *hl = M.hedge + (size_t)k * E;
    const double *ul = M.uf + (size_t)k * E;
    const size_t o = (size_t)k * N + i;
    const double mass_old = M.muf[o];
    double div = 0;
#pragma unroll
    for (int s = 0; s < 6; s++)
      if (es[s] >= 0) div += flux_coef[s] * hl[es[s]] * ul[es[s]];
    const double mass_new = mass_old - (tau * div) / area;
    M.muf[o] = mass_new;
    above += mass_new + M.div_damp * (mass_new - mass_old);
    fast_load[k] = above;
  }
  double pot = 0;
#pragma unroll
  for (int k = L - 1; k >= 0; k--) { pot += M.S[(size_t)k * N + i] * fast_load[k]; M.phi[(size_t)k * N + i] = pot; }
}

template <int L>
__device__ __forceinline__ void af_u_edge(const LayersDev &M, double tau, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const int a = g.eI[e], b = g.eJ[e];
  const double de = g.de[e], Ge = M.G[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * E + e;
    const double v = M.uf[o];
    M.accL[o] += v;
    const double *pl = M.phi + (size_t)k * N;
    M.uf[o] = v + tau * ((-(pl[b] - pl[a])) / de + M.Tp[o] + Ge);
  }
}

// stage C for air: each cell edge's flux hedge accL / n (the edge's eI cell stores it) and the floor limiter's scale
template <int L>
__device__ __forceinline__ void air_scale_cell(const LayersDev &M, const StageArgs &a, int i) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  double out[L];
#pragma unroll
  for (int k = 0; k < L; k++) out[k] = 0;
  int es[6];
  slots6(g.cellEdgeAsc, i, es);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    if (e < 0) continue;
    const bool mine = g.eI[e] == i;
    const double le = g.le[e];
#pragma unroll
    for (int k = 0; k < L; k++) {
      const size_t o = (size_t)k * E + e;
      const double F = M.hedge[o] * M.accL[o] * a.inv_n;
      if (mine) M.F[o] = F;
      const double f = F * le * a.cdt;
      if (mine) { if (f > 0) out[k] += f; }
      else if (!(f > 0)) out[k] -= f;
    }
  }
  const double A = g.areaCell[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double avail = a.h0[(size_t)k * N + i] - M.floor_;
    const double cap = (avail > 0 ? avail : 0.0) * A;
    M.scale[(size_t)k * N + i] = out[k] > cap ? cap / out[k] : 1.0;
  }
}

template <int L>
__device__ __forceinline__ void air_u_edge(const LayersDev &M, const StageArgs &a, int e) {
  const GridDev &g = M.g;
  const int E = g.E;
  const double le = g.le[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * E + e;
    if (a.Fm) a.Fm[o] = limited(M, k, e) * le * a.dt;
    a.un[o] = M.uf[o];
  }
}

// Heat of the kinetic energy removed at a cell's edges (reference kernels/layers.cu:596-621, vmix_heat): diss (J/m^2
// per edge, over the edge's kite) gives each of its two cells half of l_e d_e diss_e; the cell's share per unit area
// warms every layer of the column by the same amount per kilogram, d theta_k = q / (mu pibar_k), with pibar_k the
// layer's mass-mean Exner function from the pressures at its top and bottom. Same operation order as the reference.
template <int L>
__device__ __forceinline__ void heat_column(const GridDev &g, const double *__restrict__ h, const double *__restrict__ diss,
                                            double grav, double cp, double kap, double p0, double *__restrict__ theta, int i) {
  const int N = g.N;
  int es[6];
  slots6(g.cellEdge, i, es);
  double q = 0;
#pragma unroll
  for (int m = 0; m < 6; m++)
    if (es[m] >= 0) q += 0.5 * g.le[es[m]] * g.de[es[m]] * diss[es[m]];
  if (q == 0) return;
  q /= g.areaCell[i];
  double mass[L], mu = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    mass[k] = h[(size_t)k * N + i];
    mu += mass[k];
  }
  double pbot = 0, xtop = 0;          // pressure at the layer's bottom; (p_top / p0)^kappa
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double ptop = pbot;
    pbot = pbot + grav * mass[k];
    const double xbot = pow(pbot / p0, kap);
    const double pib = cp * (pbot * xbot - ptop * xtop) / ((kap + 1) * (pbot - ptop));
    theta[(size_t)k * N + i] += q / (mu * pib);
    xtop = xbot;
  }
}

// the interfacial stress's heat (the step's own diss) returned to theta
template <int L>
__device__ __forceinline__ void vmix_heat_cell(const LayersDev &M, const double *__restrict__ h, double *__restrict__ theta, int i) {
  heat_column<L>(M.g, h, M.diss, M.grav, M.cpa, M.kap, M.p0, theta, i);
}

template <int L>
__device__ __forceinline__ void air_gfast_cell(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ theta, int i) {
  const int N = M.g.N;
  double mu = 0;
#pragma unroll
  for (int k = 0; k < L; k++) mu += h[(size_t)k * N + i];
  int kb = L - 1;
  while (kb > 0 && h[(size_t)kb * N + i] < 2 * M.floor_) kb--;
  const double Ts = theta[(size_t)kb * N + i] * pow(M.grav * mu / M.p0, M.kap);
  double gc = M.rda * Ts / mu;
  double above = 0;
#pragma unroll
  for (int j = 0; j < L - 1; j++) {
    above += h[(size_t)j * N + i];
    const double dth = theta[(size_t)j * N + i] - theta[(size_t)(j + 1) * N + i];
    if (dth > 0) gc += dth * M.rda * pow(M.grav * above / M.p0, M.kap) * above / (mu * mu);
  }
  M.Gc[i] = gc;
}

}  // namespace fp64
}  // namespace isw
