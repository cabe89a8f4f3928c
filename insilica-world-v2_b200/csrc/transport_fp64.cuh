// Phase functions of the FCT transport step, plain FP64 form (reference kernels/fused.cu:122-241, trisk.cu:48-59).
// Rows y = tracer j * L + layer l, as the reference stacks them. A stage is an edge pass (every 3rd-order edge flux
// computed once, for all layers of a (tracer, edge)) and a cell pass that sums the fluxes in the reference's edge order
// (the reference recomputes each flux in both cells' passes); the same values and sums, with the reference's arithmetic
// (compiled with -fmad=false), so results are bit-identical:
//   HF1 / C1  stage-1 fluxes of psi; receiving mass M1 (trisk.cu:48-59), td (fused.cu:146-160), p1 (fused.cu:163-186)
//   HF2 / C2  stage-2 fluxes of p1; p2
//   A / C3    antidiffusive fluxes (fused.cu:189-194) and the Zalesak ratios (fused.cu:197-222)
//   P4        the limited update (fused.cu:225-241) into the caller's tracer arrays
// The transport's own fields (td, p1, p2, R+- per cell, the edge fluxes A per edge) are stored tracer by tracer with an
// item's layers side by side, x[(j n + i) LP + l], LP = L rounded up to even (pads 0, never summed): one gather brings
// every layer of a cell in 16-byte pairs. The caller's arrays (tracers, masses, fluxes) keep the reference's layer-major
// layout. Gathers walk a cell's six slots fully unrolled with a guard on the padded slot (no early exit); pads only
// ever trail, so the order of the sums is unchanged.
#pragma once
#include "common.cuh"

namespace isw {

struct TransportDev {
  GridDev g;
  double *td, *p1, *p2, *A, *Rp, *Rm;          // tracers x N x LP (A: tracers x E x LP), layers side by side
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

// layers per item in the transport's own fields: L rounded up to even
__host__ __device__ constexpr int lp_of(int L) { return (L + 1) & ~1; }

// offset of item i (a cell or an edge, n of them) of tracer j in a transport field of L layers
__device__ __forceinline__ size_t fx(int j, int n, int i, int L) { return ((size_t)j * n + i) * lp_of(L); }

// every layer of one item: LP / 2 16-byte loads (FP64), LP / 4 16-byte or LP / 2 8-byte loads (FP32)
template <int L>
__device__ __forceinline__ void ld_layers(const double *__restrict__ p, double v[L]) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
  for (int k = 0; k < lp_of(L) / 2; k++) {
    const double2 w = q[k];
    v[2 * k] = w.x;
    if (2 * k + 1 < L) v[2 * k + 1] = w.y;
  }
}

template <int L>
__device__ __forceinline__ void st_layers(double *__restrict__ p, const double v[L]) {
  double2 *q = reinterpret_cast<double2 *>(p);
#pragma unroll
  for (int k = 0; k < lp_of(L) / 2; k++) q[k] = make_double2(v[2 * k], 2 * k + 1 < L ? v[2 * k + 1] : 0.0);
}

template <int L>
__device__ __forceinline__ void ld_layers(const float *__restrict__ p, float v[L]) {
  constexpr int LP = lp_of(L);
  if constexpr (LP % 4 == 0) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int k = 0; k < LP / 4; k++) {
      const float4 w = q[k];
      const float x[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int m = 0; m < 4; m++)
        if (4 * k + m < L) v[4 * k + m] = x[m];
    }
  } else {
    const float2 *q = reinterpret_cast<const float2 *>(p);
#pragma unroll
    for (int k = 0; k < LP / 2; k++) {
      const float2 w = q[k];
      v[2 * k] = w.x;
      if (2 * k + 1 < L) v[2 * k + 1] = w.y;
    }
  }
}

template <int L>
__device__ __forceinline__ void st_layers(float *__restrict__ p, const float v[L]) {
  constexpr int LP = lp_of(L);
  if constexpr (LP % 4 == 0) {
    float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
    for (int k = 0; k < LP / 4; k++) {
      float x[4];
#pragma unroll
      for (int m = 0; m < 4; m++) x[m] = 4 * k + m < L ? v[4 * k + m] : 0.f;
      q[k] = make_float4(x[0], x[1], x[2], x[3]);
    }
  } else {
    float2 *q = reinterpret_cast<float2 *>(p);
#pragma unroll
    for (int k = 0; k < LP / 2; k++) q[k] = make_float2(v[2 * k], 2 * k + 1 < L ? v[2 * k + 1] : 0.f);
  }
}

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
__device__ __forceinline__ double hoflux_v(double f, const Stencil &st, double pa, double pb, double q0, double q1, double q2,
                                           double q3, double beta) {
  const double* w = st.wt;
  const double x = w[0] * pa + w[1] * pb + w[2] * q0 + w[3] * q1;
  const double y = w[4] * pb + w[5] * pa + w[6] * q2 + w[7] * q3;
  return f * (0.5 * (pa + pb) - (x + y)) + fabs(f) * ((y - x) * beta);
}

__device__ __forceinline__ double hoflux_s(double f, const double *__restrict__ ps, const Stencil &st, double pa, double pb,
                                           double beta) {
  const double q0 = ps[st.o[0]];
  const double q1 = st.o[1] == st.o[0] ? q0 : ps[st.o[1]];
  const double q2 = ps[st.o[2]];
  const double q3 = st.o[3] == st.o[2] ? q2 : ps[st.o[3]];
  return hoflux_v(f, st, pa, pb, q0, q1, q2, q3, beta);
}

// The stencil's six cells of a transport field, every layer (the opposite cells loaded once where they coincide).
template <int L, class F>
struct StencilLayers {
  F pa[L], pb[L], q0[L], q1[L], q2[L], q3[L];
};

template <int L, class F>
__device__ __forceinline__ void load_stencil_layers(const F *__restrict__ fld, int j, int N, int ea, int eb, const int o[4],
                                                    StencilLayers<L, F> &v) {
  ld_layers<L>(fld + fx(j, N, ea, L), v.pa);
  ld_layers<L>(fld + fx(j, N, eb, L), v.pb);
  ld_layers<L>(fld + fx(j, N, o[0], L), v.q0);
  ld_layers<L>(fld + fx(j, N, o[2], L), v.q2);
  if (o[1] == o[0]) {
#pragma unroll
    for (int l = 0; l < L; l++) v.q1[l] = v.q0[l];
  } else {
    ld_layers<L>(fld + fx(j, N, o[1], L), v.q1);
  }
  if (o[3] == o[2]) {
#pragma unroll
    for (int l = 0; l < L; l++) v.q3[l] = v.q2[l];
  } else {
    ld_layers<L>(fld + fx(j, N, o[3], L), v.q3);
  }
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

// P1 of the per-call order-1 step for (tracer j, cell i), every layer: td (and with order 3 p1 from fluxes recomputed
// here); with_mass: M1 formed here (tracer 0 stores it) instead of read
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
  double tdo[L], p1o[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    double mm = m1[l];
    if (with_mass) { if (j == 0) a.M1[om] = mm; }
    else mm = a.M1[om];
    tdo[l] = td[l] / mm;
    p1o[l] = s[l] / mx[l];
  }
  st_layers<L>(T.td + fx(j, N, i, L), tdo);
  if (order != 1) st_layers<L>(T.p1 + fx(j, N, i, L), p1o);
}

// the limited update of (tracer j, cell i), every layer; the cell's own ratios are loaded once, each neighbour's once
template <int L>
__device__ __forceinline__ void tr_p4(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  CellEdges c;
  load_edges(g, i, c);
  double m1[L], s[L], tdi[L], rpi[L], rmi[L];
  ld_layers<L>(T.td + fx(j, N, i, L), tdi);
  ld_layers<L>(T.Rp + fx(j, N, i, L), rpi);
  ld_layers<L>(T.Rm + fx(j, N, i, L), rmi);
#pragma unroll
  for (int l = 0; l < L; l++) {
    m1[l] = a.M1[(size_t)l * N + i];
    s[l] = tdi[l] * m1[l];
  }
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int e = c.e[q];
    if (e >= 0) {
      const bool out = c.a[q] == i;
      const int nb = out ? c.b[q] : c.a[q];
      double Av[L], rpn[L], rmn[L];
      ld_layers<L>(T.A + fx(j, E, e, L), Av);
      ld_layers<L>(T.Rp + fx(j, N, nb, L), rpn);
      ld_layers<L>(T.Rm + fx(j, N, nb, L), rmn);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double A = Av[l];
        // A > 0: min(R+ at eJ, R- at eI); else min(R+ at eI, R- at eJ)
        const double rpb = out ? rpn[l] : rpi[l], rma = out ? rmi[l] : rmn[l];
        const double rpa = out ? rpi[l] : rpn[l], rmb = out ? rmn[l] : rmi[l];
        const double cc = A > 0 ? fmin(rpb, rma) : fmin(rpa, rmb);
        if (out) s[l] -= cc * A; else s[l] += cc * A;
      }
    }
  }
#pragma unroll
  for (int l = 0; l < L; l++) a.tr[j][(size_t)l * N + i] = s[l] / m1[l];
}


// ---- The edge and cell passes of order 3 (batched and per call). The edge fluxes go to T.A, which holds the
// stage-1 fluxes, then the stage-2 fluxes, then the antidiffusive fluxes. The tracers are read in place until the
// limited update overwrites them, so no copy of them is kept. ----

// stage = 1: fluxes of the tracer itself; 2: of p1. A[j][e][l] = hoflux(f, field) for every layer.
template <int L>
__device__ __forceinline__ void tr_hf_edge(const TransportDev &T, const TrArgs &a, int stage, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  Stencil stn;
  load_stencil(g, e, stn);
  double out[L];
  if (stage == 1) {
#pragma unroll
    for (int l = 0; l < L; l++) {
      const double *p = a.tr[j] + (size_t)l * N;
      out[l] = hoflux_s(a.Fm[(size_t)l * E + e], p, stn, p[ea], p[eb], a.beta);
    }
  } else {
    StencilLayers<L, double> v;
    load_stencil_layers<L>(T.p1, j, N, ea, eb, stn.o, v);
#pragma unroll
    for (int l = 0; l < L; l++)
      out[l] = hoflux_v(a.Fm[(size_t)l * E + e], stn, v.pa[l], v.pb[l], v.q0[l], v.q1[l], v.q2[l], v.q3[l], a.beta);
  }
  st_layers<L>(T.A + fx(j, E, e, L), out);
}

// the antidiffusive flux A = hoflux(p2) - upwind(psi) of every layer of (tracer j, edge e)
template <int L>
__device__ __forceinline__ void tr_a_edge(const TransportDev &T, const TrArgs &a, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  Stencil stn;
  load_stencil(g, e, stn);
  StencilLayers<L, double> v;
  load_stencil_layers<L>(T.p2, j, N, ea, eb, stn.o, v);
  double out[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const double *p = a.tr[j] + (size_t)l * N;
    const double f = a.Fm[(size_t)l * E + e];
    out[l] = hoflux_v(f, stn, v.pa[l], v.pb[l], v.q0[l], v.q1[l], v.q2[l], v.q3[l], a.beta) - upwind_v(f, p[ea], p[eb]);
  }
  st_layers<L>(T.A + fx(j, E, e, L), out);
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
      double Av[L];
      ld_layers<L>(T.A + fx(j, E, e, L), Av);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double *p = a.tr[j] + (size_t)l * N;
        const double f = a.Fm[(size_t)l * E + e];
        const double fu = upwind_v(f, p[c.a[q]], p[c.b[q]]);
        const double hf = frac * Av[l];
        const double m = frac * f;
        if (out) { m1[l] -= f; td[l] -= fu; s[l] -= hf; mx[l] -= m; }
        else { m1[l] += f; td[l] += fu; s[l] += hf; mx[l] += m; }
      }
    }
  }
  double tdo[L], p1o[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    double mm = m1[l];
    if (with_mass) { if (j == 0) a.M1[om] = mm; }
    else mm = a.M1[om];
    tdo[l] = td[l] / mm;
    p1o[l] = s[l] / mx[l];
  }
  st_layers<L>(T.td + fx(j, N, i, L), tdo);
  st_layers<L>(T.p1 + fx(j, N, i, L), p1o);
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
      double Av[L];
      ld_layers<L>(T.A + fx(j, E, e, L), Av);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double f = a.Fm[(size_t)l * E + e];
        const double hf = frac * Av[l];
        const double m = frac * f;
        if (out) { s[l] -= hf; mx[l] -= m; } else { s[l] += hf; mx[l] += m; }
      }
    }
  }
  double p2o[L];
#pragma unroll
  for (int l = 0; l < L; l++) p2o[l] = s[l] / mx[l];
  st_layers<L>(T.p2 + fx(j, N, i, L), p2o);
}

// cell pass of stage 3: the Zalesak ratios from the antidiffusive fluxes and the bounds of psi and td
template <int L>
__device__ __forceinline__ void tr_c3(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  int es[6], nb[6];
  slots6(g.cellEdgeAsc, i, es);
  slots6(g.nbr, i, nb);
  double Pp[L], Pm[L], hi[L], lo[L], ti[L];
  ld_layers<L>(T.td + fx(j, N, i, L), ti);
#pragma unroll
  for (int l = 0; l < L; l++) {
    Pp[l] = 0;
    Pm[l] = 0;
    const double pi = a.tr[j][(size_t)l * N + i];
    hi[l] = fmax(pi, ti[l]);
    lo[l] = fmin(pi, ti[l]);
  }
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int e = es[q];
    if (e >= 0) {
      const bool out = g.eI[e] == i;
      double Av[L];
      ld_layers<L>(T.A + fx(j, E, e, L), Av);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double A = Av[l];
        if (out) { if (A > 0) Pm[l] += A; else Pp[l] -= A; }
        else { if (A > 0) Pp[l] += A; else Pm[l] -= A; }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int jn = nb[q];
    if (jn >= 0) {
      double tn[L];
      ld_layers<L>(T.td + fx(j, N, jn, L), tn);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double pn = a.tr[j][(size_t)l * N + jn];
        hi[l] = fmax(hi[l], fmax(pn, tn[l]));
        lo[l] = fmin(lo[l], fmin(pn, tn[l]));
      }
    }
  }
  double rp[L], rm[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const double m1 = a.M1[(size_t)l * N + i];
    const double qmax = (hi[l] - ti[l]) * m1, qmin = (ti[l] - lo[l]) * m1;
    rp[l] = Pp[l] > 0 ? fmin(1.0, qmax / Pp[l]) : 0.0;
    rm[l] = Pm[l] > 0 ? fmin(1.0, qmin / Pm[l]) : 0.0;
  }
  st_layers<L>(T.Rp + fx(j, N, i, L), rp);
  st_layers<L>(T.Rm + fx(j, N, i, L), rm);
}

}  // namespace fp64
}  // namespace isw
