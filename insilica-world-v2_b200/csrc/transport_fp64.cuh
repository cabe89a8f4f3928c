// Phase functions of the FCT transport step, plain FP64 form (reference kernels/fused.cu:122-241, trisk.cu:48-59).
// Rows y = tracer j * L + layer l, as the reference stacks them. One call handles one (tracer, cell) and every layer of
// it: a cell's six edges and their 3rd-order stencils are loaded once and used for all L rows of the tracer. Each
// 3rd-order edge flux is recomputed by the cell pass that sums it, with the reference's arithmetic (compiled with
// -fmad=false), and each row's sums keep the reference's edge order, so results are bit-identical.
//   P1  receiving mass M1 (trisk.cu:48-59, stored by tracer 0), td (fused.cu:146-160) and p1 (fused.cu:163-186)
//   P2  p2 (frac 1/2 from p1)
//   P3  antidiffusive fluxes A (fused.cu:189-194; stored by each edge's eI cell) and Zalesak ratios (fused.cu:197-222)
//   P4  the limited update (fused.cu:225-241) into the caller's tracer arrays
// Gathers walk a cell's six slots fully unrolled with a guard on the padded slot (no early exit), so the loads of all
// six edges can be in flight together; pads only ever trail, so the order of the sums is unchanged.
#pragma once
#include "common.cuh"

namespace isw {

struct TransportDev {
  GridDev g;
  double *psi0, *td, *p1, *p2, *A, *Rp, *Rm;   // rows x N (A rows x E); psi0 holds the tracers as they came in
  float *p1f, *p2f, *Af, *Rpf, *Rmf;           // the mixed form's FP32 stage fields, antidiffusive fluxes and ratios
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

__device__ __forceinline__ double upwind_v(double f, double pi, double pj) { return f * (f >= 0 ? pi : pj); }

// The 3rd-order stencil of an edge (csrc/grid.cu d2_stencil, reference gpu.py:86-108) is, by construction,
// [eI, eJ, o1, o2 | eJ, eI, o1', o2']: each side's cell, the other cell, and two cells opposite (the same cell twice
// on a hexagon, its weight split in halves). So an edge's flux needs the field at eI, eJ and at most four other cells;
// each distinct value is loaded once and enters the reference's expression in the reference's positions.
struct Stencil {
  int o[4];          // idx[2], idx[3], idx[6], idx[7]
  double wt[8];
};

// The tables hold 8 entries per edge (32-byte index rows, 64-byte weight rows, each table its own allocation), so the
// row is read as 8- and 16-byte vectors: a third of the L1 sector lookups of scalar loads in a thread-per-edge pass.
__device__ __forceinline__ void load_stencil(const GridDev &g, int e, Stencil &st) {
  const int2 lo = *reinterpret_cast<const int2 *>(g.d2idx + (size_t)e * 8 + 2);
  const int2 hi = *reinterpret_cast<const int2 *>(g.d2idx + (size_t)e * 8 + 6);
  st.o[0] = lo.x;
  st.o[1] = lo.y;
  st.o[2] = hi.x;
  st.o[3] = hi.y;
  const double2 *w = reinterpret_cast<const double2 *>(g.d2wt + (size_t)e * 8);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double2 v = w[q];
    st.wt[2 * q] = v.x;
    st.wt[2 * q + 1] = v.y;
  }
}

// The 3rd-order flux of an edge (reference fused.cu:131-138, FP64 form: the stencil reads the 64-bit field itself):
// f (mean - a - b) + |f| (b - a) beta, with pa = field at eI, pb = field at eJ.
__device__ __forceinline__ double hoflux_s(double f, const double *__restrict__ ps, const Stencil &st, double pa, double pb,
                                           double beta) {
  const double q0 = ps[st.o[0]];
  const double q1 = st.o[1] == st.o[0] ? q0 : ps[st.o[1]];
  const double q2 = ps[st.o[2]];
  const double q3 = st.o[3] == st.o[2] ? q2 : ps[st.o[3]];
  const double* w = st.wt;
  const double x = w[0] * pa + w[1] * pb + w[2] * q0 + w[3] * q1;
  const double y = w[4] * pb + w[5] * pa + w[6] * q2 + w[7] * q3;
  return f * (0.5 * (pa + pb) - (x + y)) + fabs(f) * ((y - x) * beta);
}

// A cell's edges in ascending edge order (cellEdgeAsc), with their two cells.
struct CellEdges {
  int e[6], a[6], b[6];
};

__device__ __forceinline__ void load_edges(const GridDev &g, int i, CellEdges &c) {
  slots6(g.cellEdgeAsc, i, c.e);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = c.e[s];
    c.a[s] = e >= 0 ? g.eI[e] : 0;
    c.b[s] = e >= 0 ? g.eJ[e] : 0;
  }
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

// P1 for (tracer j, cell i), every layer; with_mass: compute M1 here (tracer 0 stores it) instead of reading it
template <int L>
__device__ __forceinline__ void tr_p1(const TransportDev &T, const TrArgs &a, int order, bool with_mass, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  CellEdges c;
  load_edges(g, i, c);
  double m1[L], td[L], s[L], mx[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    const double m0 = a.M0[om], pi = a.tr[j][om];
    T.psi0[(size_t)(j * L + l) * N + i] = pi;
    m1[l] = m0;
    td[l] = m0 * pi;
    s[l] = m0 * pi;
    mx[l] = m0;
  }
  const double frac = 1.0 / 3.0;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int e = c.e[q];
    if (e >= 0) {
      const bool out = c.a[q] == i;
      Stencil stn;
      if (order != 1) load_stencil(g, e, stn);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double *p = a.tr[j] + (size_t)l * N;
        const double f = a.Fm[(size_t)l * E + e];
        if (with_mass) { if (out) m1[l] -= f; else m1[l] += f; }
        const double pa = p[c.a[q]], pb = p[c.b[q]];
        const double fu = upwind_v(f, pa, pb);
        if (out) td[l] -= fu; else td[l] += fu;
        if (order != 1) {
          const double hf = frac * hoflux_s(f, p, stn, pa, pb, a.beta);
          const double m = frac * f;
          if (out) { s[l] -= hf; mx[l] -= m; } else { s[l] += hf; mx[l] += m; }
        }
      }
    }
  }
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i, o = (size_t)(j * L + l) * N + i;
    double mm = m1[l];
    if (with_mass) { if (j == 0) a.M1[om] = mm; }
    else mm = a.M1[om];
    T.td[o] = td[l] / mm;
    if (order != 1) T.p1[o] = s[l] / mx[l];
  }
}

template <int L>
__device__ __forceinline__ void tr_p4(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  CellEdges c;
  load_edges(g, i, c);
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t row = (size_t)(j * L + l), om = (size_t)l * N + i;
    const double *Al = T.A + row * E;
    const double *rp = T.Rp + row * N;
    const double *rm = T.Rm + row * N;
    const double m1 = a.M1[om];
    double s = T.td[row * N + i] * m1;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int e = c.e[q];
      if (e >= 0) {
        const double A = Al[e];
        const int ea = c.a[q], eb = c.b[q];
        const double cc = A > 0 ? fmin(rp[eb], rm[ea]) : fmin(rp[ea], rm[eb]);
        if (ea == i) s -= cc * A; else s += cc * A;
      }
    }
    a.tr[j][om] = s / m1;
  }
}


// ---- The batched step's FCT: each stage as an edge pass (every 3rd-order flux computed once, for all layers of a
// (tracer, edge)) and a cell pass that sums them in the reference's edge order. The edge fluxes go to T.A (rows x E),
// which holds the stage-1 fluxes, then the stage-2 fluxes, then the antidiffusive fluxes. The tracers are read in
// place until the last pass overwrites them, so no copy psi0 is kept. Same values, same sums: bit-identical to
// tr_p1 .. tr_p4. ----

// stage = 1: fluxes of the tracer itself; 2: of p1. HF[row][e] = hoflux(f, field) for every layer.
template <int L>
__device__ __forceinline__ void tr_hf_edge(const TransportDev &T, const TrArgs &a, int stage, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  Stencil stn;
  load_stencil(g, e, stn);
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t row = (size_t)(j * L + l);
    const double *p = stage == 1 ? a.tr[j] + (size_t)l * N : T.p1 + row * N;
    T.A[row * E + e] = hoflux_s(a.Fm[(size_t)l * E + e], p, stn, p[ea], p[eb], a.beta);
  }
}

// the antidiffusive flux A = hoflux(p2) - upwind(psi) of every layer of (tracer j, edge e)
template <int L>
__device__ __forceinline__ void tr_a_edge(const TransportDev &T, const TrArgs &a, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  Stencil stn;
  load_stencil(g, e, stn);
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t row = (size_t)(j * L + l);
    const double *p = a.tr[j] + (size_t)l * N;
    const double *p2 = T.p2 + row * N;
    const double f = a.Fm[(size_t)l * E + e];
    T.A[row * E + e] = hoflux_s(f, p2, stn, p2[ea], p2[eb], a.beta) - upwind_v(f, p[ea], p[eb]);
  }
}

// cell pass of stage 1: td and p1 from the stage-1 edge fluxes; with_mass: M1 formed here (tracer 0 stores it), else
// the caller's M1 (Transport.step_many after mass_after)
template <int L>
__device__ __forceinline__ void tr_c1(const TransportDev &T, const TrArgs &a, int j, int i, bool with_mass = true) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  CellEdges c;
  load_edges(g, i, c);
  double m1[L], td[L], s[L], mx[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    const double m0 = a.M0[om], pi = a.tr[j][om];
    m1[l] = m0;
    td[l] = m0 * pi;
    s[l] = m0 * pi;
    mx[l] = m0;
  }
  const double frac = 1.0 / 3.0;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int e = c.e[q];
    if (e >= 0) {
      const bool out = c.a[q] == i;
#pragma unroll
      for (int l = 0; l < L; l++) {
        const size_t row = (size_t)(j * L + l);
        const double *p = a.tr[j] + (size_t)l * N;
        const double f = a.Fm[(size_t)l * E + e];
        const double fu = upwind_v(f, p[c.a[q]], p[c.b[q]]);
        const double hf = frac * T.A[row * E + e];
        const double m = frac * f;
        if (out) { m1[l] -= f; td[l] -= fu; s[l] -= hf; mx[l] -= m; }
        else { m1[l] += f; td[l] += fu; s[l] += hf; mx[l] += m; }
      }
    }
  }
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i, o = (size_t)(j * L + l) * N + i;
    double mm = m1[l];
    if (with_mass) { if (j == 0) a.M1[om] = mm; }
    else mm = a.M1[om];
    T.td[o] = td[l] / mm;
    T.p1[o] = s[l] / mx[l];
  }
}

// cell pass of stage 2: p2 from the stage-2 edge fluxes
template <int L>
__device__ __forceinline__ void tr_c2(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  CellEdges c;
  load_edges(g, i, c);
  double s[L], mx[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    s[l] = a.M0[om] * a.tr[j][om];
    mx[l] = a.M0[om];
  }
  const double frac = 1.0 / 2.0;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int e = c.e[q];
    if (e >= 0) {
      const bool out = c.a[q] == i;
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double f = a.Fm[(size_t)l * E + e];
        const double hf = frac * T.A[(size_t)(j * L + l) * E + e];
        const double m = frac * f;
        if (out) { s[l] -= hf; mx[l] -= m; } else { s[l] += hf; mx[l] += m; }
      }
    }
  }
#pragma unroll
  for (int l = 0; l < L; l++) T.p2[(size_t)(j * L + l) * N + i] = s[l] / mx[l];
}

// cell pass of stage 3: the Zalesak ratios from the antidiffusive fluxes and the bounds of psi and td
template <int L>
__device__ __forceinline__ void tr_c3(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  int es[6], nb[6];
  slots6(g.cellEdgeAsc, i, es);
  slots6(g.nbr, i, nb);
  bool out[6];
#pragma unroll
  for (int q = 0; q < 6; q++) out[q] = es[q] >= 0 && g.eI[es[q]] == i;
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t row = (size_t)(j * L + l);
    double Pp = 0, Pm = 0;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int e = es[q];
      if (e >= 0) {
        const double A = T.A[row * E + e];
        if (out[q]) { if (A > 0) Pm += A; else Pp -= A; }
        else { if (A > 0) Pp += A; else Pm -= A; }
      }
    }
    const double *p = a.tr[j] + (size_t)l * N;
    const double *tt = T.td + row * N;
    const double ti = tt[i];
    double hi = fmax(p[i], ti), lo = fmin(p[i], ti);
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int jn = nb[q];
      if (jn >= 0) {
        hi = fmax(hi, fmax(p[jn], tt[jn]));
        lo = fmin(lo, fmin(p[jn], tt[jn]));
      }
    }
    const double m1 = a.M1[(size_t)l * N + i];
    const double qmax = (hi - ti) * m1, qmin = (ti - lo) * m1;
    T.Rp[row * N + i] = Pp > 0 ? fmin(1.0, qmax / Pp) : 0.0;
    T.Rm[row * N + i] = Pm > 0 ? fmin(1.0, qmin / Pm) : 0.0;
  }
}

}  // namespace fp64
}  // namespace isw
