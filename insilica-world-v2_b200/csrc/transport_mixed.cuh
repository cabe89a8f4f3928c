// Phase functions of the FCT transport step, mixed form, for the batched step's edge and cell passes (the passes of
// transport_fp64.cuh, reference fused.cu:122-241) with the 3rd-order flux's curvature correction in FP32 (stencil
// weights, the stencil sums and f (a + b) - |f| (b - a) beta) and the stage fields p1, p2, the antidiffusive fluxes A
// and the ratios R+- stored in FP32, as the reference's
// mixed form keeps its stencil weights and field copy 32-bit (gpu.py:77, transport.py:28). Tracer masses stay FP64:
// the upwind fluxes, the mean-value part of the 3rd-order flux f (p_I + p_J) / 2, every cell sum, td, the bounds and the
// limited update. Each edge's flux enters both of its cells with the same value (the passes compute it from the same
// operands in the same order, and A is rounded to FP32 once, before its use in either the ratios or the update), so the
// tracer mass moves between cells exactly as in FP64.
#pragma once
#include "common.cuh"
#include "transport_fp64.cuh"

namespace isw {
namespace mixed {

struct Stencil32 {
  int o[4];
  float wt[8];
};

__device__ __forceinline__ void load_stencil(const GridDev &g, int e, Stencil32 &st) {
  const int2 lo = *reinterpret_cast<const int2 *>(g.d2idx + (size_t)e * 8 + 2);
  const int2 hi = *reinterpret_cast<const int2 *>(g.d2idx + (size_t)e * 8 + 6);
  st.o[0] = lo.x;
  st.o[1] = lo.y;
  st.o[2] = hi.x;
  st.o[3] = hi.y;
  const float4 *w = reinterpret_cast<const float4 *>(g.d2wt32 + (size_t)e * 8);
  const float4 a = w[0], b = w[1];
  st.wt[0] = a.x; st.wt[1] = a.y; st.wt[2] = a.z; st.wt[3] = a.w;
  st.wt[4] = b.x; st.wt[5] = b.y; st.wt[6] = b.z; st.wt[7] = b.w;
}

// f (mean - x - y) + |f| (y - x) beta: the mean part in FP64, the curvature correction in FP32.
template <class T>
__device__ __forceinline__ double hoflux_v(double f, const Stencil32 &st, T pa, T pb, float q0, float q1, float q2, float q3,
                                           float beta) {
  const float fa = (float)pa, fb = (float)pb;
  const float *w = st.wt;
  const float x = w[0] * fa + w[1] * fb + w[2] * q0 + w[3] * q1;
  const float y = w[4] * fb + w[5] * fa + w[6] * q2 + w[7] * q3;
  const float ff = (float)f;
  const float corr = fabsf(ff) * ((y - x) * beta) - ff * (x + y);
  return f * (0.5 * ((double)pa + (double)pb)) + (double)corr;
}

template <class T>
__device__ __forceinline__ double hoflux(double f, const T *__restrict__ ps, const Stencil32 &st, T pa, T pb, float beta) {
  const float q0 = (float)ps[st.o[0]];
  const float q1 = st.o[1] == st.o[0] ? q0 : (float)ps[st.o[1]];
  const float q2 = (float)ps[st.o[2]];
  const float q3 = st.o[3] == st.o[2] ? q2 : (float)ps[st.o[3]];
  return hoflux_v(f, st, pa, pb, q0, q1, q2, q3, beta);
}

// the limited update of (tracer j, cell i), every layer (FP32 ratios and antidiffusive fluxes, FP64 sums)
template <int L>
__device__ __forceinline__ void tr_p4(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  fp64::CellEdges c;
  fp64::load_edges(g, i, c);
  double m1[L], s[L], tdi[L];
  float rpi[L], rmi[L];
  ld_layers<L>(T.td + fx(j, N, i, L), tdi);
  ld_layers<L>(T.Rpf + fx(j, N, i, L), rpi);
  ld_layers<L>(T.Rmf + fx(j, N, i, L), rmi);
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
      float Av[L], rpn[L], rmn[L];
      ld_layers<L>(T.Af + fx(j, E, e, L), Av);
      ld_layers<L>(T.Rpf + fx(j, N, nb, L), rpn);
      ld_layers<L>(T.Rmf + fx(j, N, nb, L), rmn);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const float A = Av[l];
        const float rpb = out ? rpn[l] : rpi[l], rma = out ? rmi[l] : rmn[l];
        const float rpa = out ? rpi[l] : rpn[l], rmb = out ? rmn[l] : rmi[l];
        const float cc = A > 0 ? fminf(rpb, rma) : fminf(rpa, rmb);
        const double fl = (double)cc * (double)A;
        if (out) s[l] -= fl; else s[l] += fl;
      }
    }
  }
#pragma unroll
  for (int l = 0; l < L; l++) a.tr[j][(size_t)l * N + i] = s[l] / m1[l];
}


// ---- The batched step's FCT in the mixed form, as edge passes and cell passes (see transport_fp64.cuh): the stage
// fluxes of the edge passes are stored in FP64 (T.A), the antidiffusive fluxes rounded to FP32 once (T.Af). ----

template <int L>
__device__ __forceinline__ void tr_hf_edge(const TransportDev &T, const TrArgs &a, int stage, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  const float beta = (float)a.beta;
  Stencil32 stn;
  load_stencil(g, e, stn);
  double out[L];
  if (stage == 1) {
#pragma unroll
    for (int l = 0; l < L; l++) {
      const double *p = a.tr[j] + (size_t)l * N;
      out[l] = hoflux(a.Fm[(size_t)l * E + e], p, stn, p[ea], p[eb], beta);
    }
  } else {
    fp64::StencilLayers<L, float> v;
    fp64::load_stencil_layers<L>(T.p1f, j, N, ea, eb, stn.o, v);
#pragma unroll
    for (int l = 0; l < L; l++)
      out[l] = hoflux_v(a.Fm[(size_t)l * E + e], stn, v.pa[l], v.pb[l], v.q0[l], v.q1[l], v.q2[l], v.q3[l], beta);
  }
  st_layers<L>(T.A + fx(j, E, e, L), out);
}

template <int L>
__device__ __forceinline__ void tr_a_edge(const TransportDev &T, const TrArgs &a, int j, int e) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  const float beta = (float)a.beta;
  Stencil32 stn;
  load_stencil(g, e, stn);
  fp64::StencilLayers<L, float> v;
  fp64::load_stencil_layers<L>(T.p2f, j, N, ea, eb, stn.o, v);
  float out[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const double *p = a.tr[j] + (size_t)l * N;
    const double f = a.Fm[(size_t)l * E + e];
    out[l] = (float)(hoflux_v(f, stn, v.pa[l], v.pb[l], v.q0[l], v.q1[l], v.q2[l], v.q3[l], beta) -
                     fp64::upwind_v(f, p[ea], p[eb]));
  }
  st_layers<L>(T.Af + fx(j, E, e, L), out);
}

template <int L>
__device__ __forceinline__ void tr_c1(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  fp64::CellEdges c;
  fp64::load_edges(g, i, c);
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
        const double fu = fp64::upwind_v(f, p[c.a[q]], p[c.b[q]]);
        const double hf = frac * Av[l];
        const double m = frac * f;
        if (out) { m1[l] -= f; td[l] -= fu; s[l] -= hf; mx[l] -= m; }
        else { m1[l] += f; td[l] += fu; s[l] += hf; mx[l] += m; }
      }
    }
  }
  double tdo[L];
  float p1o[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const size_t om = (size_t)l * N + i;
    if (j == 0) a.M1[om] = m1[l];
    tdo[l] = td[l] / m1[l];
    p1o[l] = (float)(s[l] / mx[l]);
  }
  st_layers<L>(T.td + fx(j, N, i, L), tdo);
  st_layers<L>(T.p1f + fx(j, N, i, L), p1o);
}

template <int L>
__device__ __forceinline__ void tr_c2(const TransportDev &T, const TrArgs &a, int j, int i) {
  const GridDev &g = T.g;
  const int N = g.N, E = g.E;
  fp64::CellEdges c;
  fp64::load_edges(g, i, c);
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
  float p2o[L];
#pragma unroll
  for (int l = 0; l < L; l++) p2o[l] = (float)(s[l] / mx[l]);
  st_layers<L>(T.p2f + fx(j, N, i, L), p2o);
}

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
      float Av[L];
      ld_layers<L>(T.Af + fx(j, E, e, L), Av);
#pragma unroll
      for (int l = 0; l < L; l++) {
        const double A = (double)Av[l];
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
  float rp[L], rm[L];
#pragma unroll
  for (int l = 0; l < L; l++) {
    const double m1 = a.M1[(size_t)l * N + i];
    const double qmax = (hi[l] - ti[l]) * m1, qmin = (ti[l] - lo[l]) * m1;
    rp[l] = Pp[l] > 0 ? (float)fmin(1.0, qmax / Pp[l]) : 0.f;
    rm[l] = Pm[l] > 0 ? (float)fmin(1.0, qmin / Pm[l]) : 0.f;
  }
  st_layers<L>(T.Rpf + fx(j, N, i, L), rp);
  st_layers<L>(T.Rmf + fx(j, N, i, L), rm);
}

}  // namespace mixed
}  // namespace isw
