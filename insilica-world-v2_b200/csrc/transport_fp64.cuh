// Phase functions of the FCT transport step, plain FP64 form (reference kernels/fused.cu:122-241, trisk.cu:48-59): one
// call per (row, cell), rows y = tracer j * L + layer l. Each 3rd-order edge flux is recomputed by the cell pass that
// sums it, with the reference's arithmetic (compiled with -fmad=false), so results are bit-identical.
//   P1  receiving mass M1 (trisk.cu:48-59, stored by the j = 0 rows), td (fused.cu:146-160) and p1 (fused.cu:163-186)
//   P2  p2 (frac 1/2 from p1)
//   P3  antidiffusive fluxes A (fused.cu:189-194; stored by each edge's eI cell) and Zalesak ratios (fused.cu:197-222)
//   P4  the limited update (fused.cu:225-241) into the caller's tracer arrays
#pragma once
#include "common.cuh"

namespace isw {

struct TransportDev {
  GridDev g;
  double *psi0, *td, *p1, *p2, *A, *Rp, *Rm;   // rows x N (A rows x E); psi0 holds the tracers as they came in
};

// Per-call arguments: the masses, the fluxes and the caller's tracer arrays.
struct TrArgs {
  const double *M0, *Fm;
  double *M1;
  double *tr[TRMAX];
  int L, rows;
  double beta;
};

namespace fp64 {

__device__ __forceinline__ double upwind(const double *__restrict__ Fml, const double *__restrict__ p, const int *eI, const int *eJ,
                                         int e) {
  const double f = Fml[e];
  return f * (f >= 0 ? p[eI[e]] : p[eJ[e]]);
}

// reference fused.cu:131-138, FP64 form (the stencil reads the 64-bit field itself)
__device__ __forceinline__ double hoflux(const GridDev &g, const double *__restrict__ Fml, const double *__restrict__ ps, int e,
                                         double beta) {
  const double f = Fml[e];
  const int o = e * 8;
  const int *idx = g.d2idx;
  const double *wt = g.d2wt;
  const double a = wt[o] * ps[idx[o]] + wt[o + 1] * ps[idx[o + 1]] + wt[o + 2] * ps[idx[o + 2]] + wt[o + 3] * ps[idx[o + 3]];
  const double b = wt[o + 4] * ps[idx[o + 4]] + wt[o + 5] * ps[idx[o + 5]] + wt[o + 6] * ps[idx[o + 6]] + wt[o + 7] * ps[idx[o + 7]];
  return f * (0.5 * (ps[g.eI[e]] + ps[g.eJ[e]]) - (a + b)) + fabs(f) * ((b - a) * beta);
}

// reference trisk.cu:48-59
__device__ __forceinline__ double mass_cell(const GridDev &g, const double *__restrict__ M0, const double *__restrict__ Fml, int l, int i) {
  double m = M0[(size_t)l * g.N + i];
  for (int k = 0; k < 6; k++) {
    const int e = g.cellEdgeAsc[i * 6 + k];
    if (e < 0) break;
    if (g.eI[e] == i) m -= Fml[e]; else m += Fml[e];
  }
  return m;
}

// P1 for (row y, cell i); with_mass: compute M1 here (rows of tracer 0 store it) instead of reading it
__device__ __forceinline__ void tr_p1(const TransportDev &T, const TrArgs &a, int order, bool with_mass, int y, int i) {
  const GridDev &g = T.g;
  const int l = y % a.L, j = y / a.L;
  const size_t o = (size_t)y * g.N + i, om = (size_t)l * g.N + i;
  const double *p = a.tr[j] + (size_t)l * g.N;
  const double *Fml = a.Fm + (size_t)l * g.E;
  double m1;
  if (with_mass) {
    m1 = mass_cell(g, a.M0, Fml, l, i);
    if (j == 0) a.M1[om] = m1;
  } else {
    m1 = a.M1[om];
  }
  const double pi = p[i];
  T.psi0[o] = pi;
  const double m0 = a.M0[om];
  double td = m0 * pi;
  double s = m0 * pi, mx = m0;
  const double frac = 1.0 / 3.0;
  for (int k = 0; k < 6; k++) {
    const int e = g.cellEdgeAsc[i * 6 + k];
    if (e < 0) break;
    const bool out = g.eI[e] == i;
    const double fu = upwind(Fml, p, g.eI, g.eJ, e);
    if (out) td -= fu; else td += fu;
    if (order != 1) {
      const double f = frac * hoflux(g, Fml, p, e, a.beta);
      const double m = frac * Fml[e];
      if (out) { s -= f; mx -= m; } else { s += f; mx += m; }
    }
  }
  T.td[o] = td / m1;
  if (order != 1) T.p1[o] = s / mx;
}

__device__ __forceinline__ void tr_p2(const TransportDev &T, const TrArgs &a, int y, int i) {
  const GridDev &g = T.g;
  const int l = y % a.L;
  const size_t o = (size_t)y * g.N + i, om = (size_t)l * g.N + i;
  const double *p1 = T.p1 + (size_t)y * g.N;
  const double *Fml = a.Fm + (size_t)l * g.E;
  const double frac = 1.0 / 2.0;
  double s = a.M0[om] * T.psi0[o], mx = a.M0[om];
  for (int k = 0; k < 6; k++) {
    const int e = g.cellEdgeAsc[i * 6 + k];
    if (e < 0) break;
    const double f = frac * hoflux(g, Fml, p1, e, a.beta);
    const double m = frac * Fml[e];
    if (g.eI[e] == i) { s -= f; mx -= m; } else { s += f; mx += m; }
  }
  T.p2[o] = s / mx;
}

__device__ __forceinline__ void tr_p3(const TransportDev &T, const TrArgs &a, int y, int i) {
  const GridDev &g = T.g;
  const int l = y % a.L;
  const double *p = T.psi0 + (size_t)y * g.N;
  const double *tt = T.td + (size_t)y * g.N;
  const double *p2 = T.p2 + (size_t)y * g.N;
  const double *Fml = a.Fm + (size_t)l * g.E;
  double hi = fmax(p[i], tt[i]), lo = fmin(p[i], tt[i]);
  for (int k = 0; k < 6; k++) {
    const int j = g.nbr[i * 6 + k];
    if (j < 0) break;
    hi = fmax(hi, fmax(p[j], tt[j]));
    lo = fmin(lo, fmin(p[j], tt[j]));
  }
  const double m1 = a.M1[(size_t)l * g.N + i];
  const double qmax = (hi - tt[i]) * m1, qmin = (tt[i] - lo) * m1;
  double Pp = 0, Pm = 0;
  for (int k = 0; k < 6; k++) {
    const int e = g.cellEdgeAsc[i * 6 + k];
    if (e < 0) break;
    const double A = hoflux(g, Fml, p2, e, a.beta) - upwind(Fml, p, g.eI, g.eJ, e);
    if (g.eI[e] == i) {
      T.A[(size_t)y * g.E + e] = A;
      if (A > 0) Pm += A; else Pp -= A;
    } else {
      if (A > 0) Pp += A; else Pm -= A;
    }
  }
  T.Rp[(size_t)y * g.N + i] = Pp > 0 ? fmin(1.0, qmax / Pp) : 0.0;
  T.Rm[(size_t)y * g.N + i] = Pm > 0 ? fmin(1.0, qmin / Pm) : 0.0;
}

__device__ __forceinline__ void tr_p4(const TransportDev &T, const TrArgs &a, int y, int i) {
  const GridDev &g = T.g;
  const int l = y % a.L, j = y / a.L;
  const size_t o = (size_t)y * g.N + i, om = (size_t)l * g.N + i;
  const double *Al = T.A + (size_t)y * g.E;
  const double *rp = T.Rp + (size_t)y * g.N;
  const double *rm = T.Rm + (size_t)y * g.N;
  const double m1 = a.M1[om];
  double s = T.td[o] * m1;
  for (int k = 0; k < 6; k++) {
    const int e = g.cellEdgeAsc[i * 6 + k];
    if (e < 0) break;
    const double A = Al[e];
    const int ea = g.eI[e], eb = g.eJ[e];
    const double c = A > 0 ? fmin(rp[eb], rm[ea]) : fmin(rp[ea], rm[eb]);
    if (ea == i) s -= c * A; else s += c * A;
  }
  a.tr[j][(size_t)l * g.N + i] = s / m1;
}

}  // namespace fp64
}  // namespace isw
