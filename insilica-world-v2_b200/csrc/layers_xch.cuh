// The between-step exchange hook (reference layers.py:214-232, Layers.exchange; kernels/layers.cu:452-545): thickness
// wx (L - 1 rows, positive upward across the interface below layer k) moves between neighbouring layers with its
// tracer (upwind) and momentum, conservatively; for air the kinetic energy the momentum mixing removes (and the step's
// nabla^4 loss) returns as heat, and a nearly empty layer takes its neighbours' wind. Plain FP64, the reference's
// operation order (compiled with -fmad=false): results are bit-identical to the reference's.
#pragma once
#include "common.cuh"

namespace isw {
namespace fp64 {

// cells: h, M and the tracer psi of every layer (xch_cell). seq: the passes in the order water moves through the
// column, each donor's tracer as it stands then.
template <int L>
__device__ __forceinline__ void xch_cell(const LayersDev &M, const double *__restrict__ wx, double *__restrict__ h,
                                         double *__restrict__ Mm, double *__restrict__ psi, int seq, int i) {
  const int N = M.g.N;
  const double A = M.g.areaCell[i];
  if (seq) {
    double m[L], t[L];
#pragma unroll
    for (int k = 0; k < L; k++) {
      const size_t o = (size_t)k * N + i;
      m[k] = Mm[o];
      t[k] = Mm[o] * psi[o];
    }
    for (int pass = 0; pass < 2; pass++)
      for (int n = 0; n + 1 < L; n++) {
        const int k = pass == 0 ? L - 2 - n : n;
        const double v = wx[(size_t)k * N + i];
        if (pass == 0 ? !(v > 0) : !(v < 0)) continue;
        const int d = v > 0 ? k + 1 : k;
        const double vol = v * A, p = t[d] / m[d];
        m[k] += vol;
        m[k + 1] -= vol;
        t[k] += vol * p;
        t[k + 1] -= vol * p;
      }
#pragma unroll
    for (int k = 0; k < L; k++) {
      const size_t o = (size_t)k * N + i;
      h[o] = h[o] + (m[k] - Mm[o]) / A;
      Mm[o] = m[k];
      psi[o] = t[k] / m[k];
    }
    return;
  }
  double tr[L], dm[L];
#pragma unroll
  for (int k = 0; k < L; k++) { tr[k] = 0; dm[k] = 0; }
#pragma unroll
  for (int k = 0; k + 1 < L; k++) {
    const double v = wx[(size_t)k * N + i];
    const double p = v > 0 ? psi[(size_t)(k + 1) * N + i] : psi[(size_t)k * N + i];
    const double vol = v * A;
    dm[k] += vol;
    dm[k + 1] -= vol;
    tr[k] += vol * p;
    tr[k + 1] -= vol * p;
  }
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * N + i;
    const double m1 = Mm[o] + dm[k];
    psi[o] = (Mm[o] * psi[o] + tr[k]) / m1;
    Mm[o] = m1;
    h[o] = h[o] + dm[k] / A;
  }
}

// edges: every layer's wind with the edge thicknesses before the exchange (hold), column momentum h_e u conserved
// (xch_edge). diss (or null) receives the kinetic energy removed, with nu4dt sum h_e u lap4 when lap4 is given; hthin
// > 0: a nearly empty layer moves toward its neighbours' mass-weighted wind.
template <int L>
__device__ __forceinline__ void xch_edge(const LayersDev &M, const double *__restrict__ wx, const double *__restrict__ hold,
                                         double *__restrict__ u, double *__restrict__ diss, const double *__restrict__ lap4,
                                         double nu4dt, double hthin, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const int ia = g.eI[e], ib = g.eJ[e];
  const double floor_ = M.floor_;
  double mom[L], hn[L];
  double k0 = 0, v4 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double he = 0.5 * (hold[(size_t)k * N + ia] + hold[(size_t)k * N + ib]);
    const double uk = u[(size_t)k * E + e];
    mom[k] = he * uk;
    hn[k] = he;
    k0 += he * uk * uk;
    if (lap4) v4 += he * uk * lap4[(size_t)k * E + e];
  }
  for (int pass = 0; pass < 2; pass++)
    for (int n = 0; n + 1 < L; n++) {
      const int k = pass == 0 ? L - 2 - n : n;
      const double v = 0.5 * (wx[(size_t)k * N + ia] + wx[(size_t)k * N + ib]);
      if (pass == 0 ? !(v > 0) : !(v < 0)) continue;
      const int d = v > 0 ? k + 1 : k;
      const double ud = hn[d] > floor_ ? mom[d] / hn[d] : u[(size_t)d * E + e];
      mom[k] += v * ud;
      mom[k + 1] -= v * ud;
      hn[k] += v;
      hn[k + 1] -= v;
    }
  double un[L];
#pragma unroll
  for (int k = 0; k < L; k++) un[k] = mom[k] / hn[k];
  if (hthin > 0)
    for (int k = 0; k < L; k++) {
      const double hm = fmin(hold[(size_t)k * N + ia], hold[(size_t)k * N + ib]);
      if (hm >= hthin) continue;
      double w = (hthin - hm) / (hthin - floor_);
      if (w > 1) w = 1;
      double hs = 0, ms = 0;
      if (k > 0) { hs += hn[k - 1]; ms += hn[k - 1] * un[k - 1]; }
      if (k + 1 < L) { hs += hn[k + 1]; ms += hn[k + 1] * un[k + 1]; }
      if (hs <= 0) continue;
      w = fmin(w, hs / (hn[k] + hs));
      const double du = w * (ms / hs - un[k]);
      un[k] += du;
      const double dn = hn[k] * du / hs;
      if (k > 0) un[k - 1] -= dn;
      if (k + 1 < L) un[k + 1] -= dn;
    }
  double k1 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    u[(size_t)k * E + e] = un[k];
    k1 += hn[k] * un[k] * un[k];
  }
  if (diss) diss[e] = 0.5 * (k0 - k1) + nu4dt * v4;
  if (M.wall && M.wall[e] == 0)    // walls: the exchange's wind masked after it (reference layers.py:226)
    for (int k = 0; k < L; k++) u[(size_t)k * E + e] = 0.0;
}

}  // namespace fp64
}  // namespace isw
