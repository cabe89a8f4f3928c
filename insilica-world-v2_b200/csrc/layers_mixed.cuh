// Phase functions of the time-split RK3 step, mixed form: the same phases as layers_fp64.cuh (reference layers.py:129-212),
// with momentum, the TRiSK operators and the slow tendencies in FP32 and the quantities whose size dwarfs their change
// in FP64, so that FP32 rounding only ever lands on small numbers:
//   FP64  thicknesses h (stage and final) and every sum that updates them, the limiter's bound, the Montgomery
//         potential B, the free surface eta0, the barotropic wind at the step start ubar0 and the sub-step sum acc, the
//         final wind u = u0 + dt T' + (ubar - ubar0), the interfacial stress (vmix);
//   FP32  the stage winds u1, u2 (and u's FP32 copy for stage 1), q, the packed neighbour record, the PV flux, KE, the
//         Laplacians, T' and the column force, H_e, the fast loop's state, and the stored layer fluxes F and limiter
//         factors (computed in FP64, each stored once per edge or cell).
// The fast loop runs in deviation form: deta = eta - eta0 and dub = ubar - ubar0, both zero at each stage's start and
// small, with eta0's gradient folded into the column force once per stage (G' = G - (Gc_J eta0_J - Gc_I eta0_I) / d_e)
// and ubar0's divergence once per cell (c0 = sum sign l_e H_e ubar0); acc sums dub in FP64, so the mean barotropic wind
// is ubar0 + acc / n. Division by a fixed grid quantity multiplies by its stored reciprocal (as the reference's mixed
// form does, layers.cu:15-21). Mass stays exact to FP64 rounding: each edge's flux is one FP64 value used by both cells.
#pragma once
#include "common.cuh"
#include "layers_fp64.cuh"

namespace isw {
namespace mixed {

// Stage arguments of the mixed form: stage winds in FP32; the final stage writes the caller's FP64 u.
struct MStageArgs {
  const double *hs, *h0, *u0;
  const float *us, *u0f;
  double *hn, *un, *Fm;        // un: the final stage only
  float *unf;                  // stages 1 and 2
  double cdt, dt, inv_n;
  float tau;
  int n;
};

// ---- init: u's FP32 copy with the column wind ubar0 (FP64), and the Laplacian passes in FP32 ----
template <int L>
__device__ __forceinline__ void ubar0_edge(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u, int e) {
  const int N = M.g.N, E = M.g.E;
  const int a = M.g.eI[e], b = M.g.eJ[e];
  double H = 0, U = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double he = 0.5 * (h[(size_t)k * N + a] + h[(size_t)k * N + b]);
    const double ue = u[(size_t)k * E + e];
    H += he;
    U += he * ue;
    M.u32[(size_t)k * E + e] = (float)ue;
  }
  M.ub0[e] = U / H;
}

template <int L, class T>
__device__ __forceinline__ void div_cell(const LayersDev &M, const T *__restrict__ u, int i) {
  const GridDev &g = M.g;
  int es[6];
  float c[6];
  slots6(g.cellEdge, i, es);
  int sg[6];
  signs6(g.cellSign, i, sg);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    c[s] = e >= 0 ? (float)sg[s] * g.le32[e] : 0.f;
  }
  const float rA = g.rA32[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const T *ul = u + (size_t)k * g.E;
    float s = 0;
#pragma unroll
    for (int t = 0; t < 6; t++)
      if (es[t] >= 0) s += c[t] * (float)ul[es[t]];
    M.D1f[(size_t)k * g.N + i] = s * rA;
  }
}

template <int L, class T>
__device__ __forceinline__ void curl_vertex(const LayersDev &M, const T *__restrict__ u, int v) {
  const GridDev &g = M.g;
  int es[3];
  float c[3];
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const int e = g.vEdge[v * 3 + s];
    es[s] = e;
    c[s] = (float)g.vEdgeSign[v * 3 + s] * g.de32[e];
  }
  const float rA = g.rAV32[v];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const T *ul = u + (size_t)k * g.E;
    float z = 0;
#pragma unroll
    for (int s = 0; s < 3; s++) z += c[s] * (float)ul[es[s]];
    M.Z1f[(size_t)k * g.NV + v] = z * rA;
  }
}

template <int L>
__device__ __forceinline__ void lap_edge(const LayersDev &M, float *__restrict__ out, int e) {
  const GridDev &g = M.g;
  const int a = g.eI[e], b = g.eJ[e], v1 = g.ev1[e], v2 = g.ev2[e];
  const float rde = g.rde32[e], rle = g.rle32[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const float *Dl = M.D1f + (size_t)k * g.N;
    const float *Zl = M.Z1f + (size_t)k * g.NV;
    out[(size_t)k * g.E + e] = (Dl[b] - Dl[a]) * rde - (Zl[v2] - Zl[v1]) * rle;
  }
}

// ---- stage phase A: B (FP64 Montgomery part plus FP32 kinetic energy), q (FP32) ----
template <int L>
__device__ __forceinline__ void bern_cell(const LayersDev &M, const double *__restrict__ h, const float *__restrict__ u, int i) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  double z[L];
  double s = M.b[i];
#pragma unroll
  for (int k = L - 1; k >= 0; k--) { s += h[(size_t)k * N + i]; z[k] = s; }
  int es[6];
  float c[6];
  slots6(g.cellEdge, i, es);
#pragma unroll
  for (int t = 0; t < 6; t++) {
    const int e = es[t];
    c[t] = e >= 0 ? g.le32[e] * g.de32[e] * 0.25f : 0.f;
  }
  const float rA = g.rA32[i];
  double Mp = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    if (k > 0) Mp += M.gp[k - 1] * z[k];
    const float *ul = u + (size_t)k * E;
    float ke = 0;
#pragma unroll
    for (int t = 0; t < 6; t++)
      if (es[t] >= 0) {
        const float ue = ul[es[t]];
        ke += c[t] * ue * ue;
      }
    M.B[(size_t)k * N + i] = Mp + (double)(ke * rA);
  }
  M.deta[i] = 0.f;                       // the grid-wide fast loop's start (tiles start from zero themselves)
}

template <int L>
__device__ __forceinline__ void pv_vertex(const LayersDev &M, const double *__restrict__ h, const float *__restrict__ u, int v) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E, NV = g.NV;
  int cs[3], es[3];
  float kw[3], c[3];
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const int cc = g.vCell[v * 3 + s];
    cs[s] = cc;
    kw[s] = g.kite32[cc * 6 + g.vSlot[v * 3 + s]];
    const int e = g.vEdge[v * 3 + s];
    es[s] = e;
    c[s] = (float)g.vEdgeSign[v * 3 + s] * g.de32[e];
  }
  const float rAv = g.rAV32[v], f = (float)M.fV[v];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *hl = h + (size_t)k * N;
    const float *ul = u + (size_t)k * E;
    float hv = 0, z = 0;
#pragma unroll
    for (int s = 0; s < 3; s++) hv += kw[s] * (float)hl[cs[s]];
#pragma unroll
    for (int s = 0; s < 3; s++) z += c[s] * ul[es[s]];
    M.q32[(size_t)k * NV + v] = (z * rAv + f) / (hv * rAv);
  }
}

// ---- stage phase E: the packed neighbour record (h_e, u, q_e) per edge and layer; fast-loop accumulators to zero ----
template <int L>
__device__ __forceinline__ void edge_hq(const LayersDev &M, const double *__restrict__ h, const float *__restrict__ u, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E, NV = g.NV;
  const int a = g.eI[e], b = g.eJ[e], v1 = g.ev1[e], v2 = g.ev2[e];
  float4 *pp = M.pk4 + (size_t)e * L;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const float hv = (float)(0.5 * (h[(size_t)k * N + a] + h[(size_t)k * N + b]));
    const float qv = 0.5f * (M.q32[(size_t)k * NV + v1] + M.q32[(size_t)k * NV + v2]);
    pp[k] = make_float4(hv, u[(size_t)k * E + e], qv, 0.f);
  }
  M.dub[e] = 0.f;
  M.acc[e] = 0.0;
}

// ---- stage phase S: slow tendencies in FP32; the pressure gradient from the FP64 B ----
// Copy into shared memory the packed records (every layer's float4) of the distinct edges named by the rows of edge
// block c; every thread of the block takes part, the caller synchronises before reading.
template <int L>
__device__ __forceinline__ void stage_pk4(const LayersDev &M, int c, float4 *stg) {
  const int b0 = M.g.sOff[c], n = (M.g.sOff[c + 1] - b0) * L;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int r = q / L;
    stg[q] = M.pk4[(size_t)M.g.sList[b0 + r] * L + (q - r * L)];
  }
}

// STG: the neighbours' records come from `stg` (stage_pk4) instead of M.pk4; the same values in the same order.
template <int L, bool STG = false>
__device__ __forceinline__ void slow_edge(const LayersDev &M, const float *__restrict__ u, double dts, int e,
                                          const float4 *stg = nullptr) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  float he[L], cap[L], qf[L], Q[L];
  const float thin = (float)M.thin;
  const float4 *pe = M.pk4 + (size_t)e * L;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const float4 p = pe[k];
    he[k] = p.x;
    cap[k] = thin * p.x;
    qf[k] = p.z;
    Q[k] = 0.f;
  }
  const int cnt = g.eoeStart[e + 1] - g.eoeStart[e];
  int ix[EOE_MAX];
  float wv[EOE_MAX];
  if (STG) {
    trisk_loc(g, e, ix);
    trisk_weights(g, e, wv);
  } else {
    trisk_row(g, e, ix, wv);
  }
#pragma unroll
  for (int t = 0; t < EOE_MAX; t++) {
    if (t < cnt) {
      const float wm = wv[t];
      const float4 *pp = (STG ? stg : M.pk4) + (size_t)ix[t] * L;
#pragma unroll
      for (int k = 0; k < L; k++) {
        const float4 p = pp[k];
        Q[k] += wm * (fminf(p.x, cap[k]) * p.y) * 0.5f * (qf[k] + p.z);
      }
    }
  }
  const int a = g.eI[e], b = g.eJ[e];
  const double rde = g.rde[e];
  const float fdts = (float)dts, flo = (float)M.floor_, nu4 = (float)M.nu4;
  float T[L];
  float H = 0, U = 0, GT = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const float ue = u[(size_t)k * E + e];
    const double *Bl = M.B + (size_t)k * N;
    float d = Q[k] - (float)((Bl[b] - Bl[a]) * rde) - (float)M.drag[k] * ue;
    const float ck = (float)M.stress[k];
    if (ck != 0.f) {
      const float r = ck / fmaxf(he[k], flo);
      const float rd = r * fdts;
      d -= (rd > 1e-8f ? -expm1f(-rd) / fdts : r) * ue;     // exact exponential decay over the stage
    }
    if (nu4 != 0.f) d -= nu4 * M.L2f[(size_t)k * E + e];
    T[k] = d;
    H += he[k];
    U += he[k] * ue;
  }
#pragma unroll
  for (int k = 0; k < L; k++) GT += he[k] * T[k];
  const float gm = GT / H;
#pragma unroll
  for (int k = 0; k < L; k++) M.Tp32[(size_t)k * E + e] = T[k] - gm;
  const double gb = (M.Gc[b] * M.eta0[b] - M.Gc[a] * M.eta0[a]) * rde;   // eta0's gradient, FP64
  const float G = (float)((double)gm - gb);
  M.G32[e] = G;
  M.Gr32[e] = make_float2(G, (float)rde);
  M.He32[e] = H;
  M.ubs32[e] = U / H;
}

// The grid-wide fast loop's per-item roundings, written out (explicit fused multiply-adds) so that every form of the
// loop that uses them (item by item, over wide chunks, the persistent loop) gives the same bits: an edge's new dub, a
// cell's new deta and its Y = Gc (deta + gamma (deta - deta_prev)).
__device__ __forceinline__ float bt_u_new(float v, float tau, float G, float yi, float yj, float rde) {
  return __fmaf_rn(tau, __fmaf_rn(-__fsub_rn(yj, yi), rde, G), v);
}
__device__ __forceinline__ float bt_eta_new(float d0, float tau, float div) {   // div already over the cell's area
  return __fmaf_rn(-tau, div, d0);
}
__device__ __forceinline__ float bt_y_new(float gc, float gam, float dn, float d0) {
  return __fmul_rn(gc, __fmaf_rn(gam, __fsub_rn(dn, d0), dn));
}

// The sub-steps' sum of dub at an edge without a per-edge running sum. With dub_0 = 0 and dub_{j+1} = dub_j +
// tau (G - (Y_j[J] - Y_j[I]) / d_e), the sum over j < n of dub_j is
//     tau (G n (n - 1) / 2 - (W[J] - W[I]) / d_e),   W = sum over j <= n - 2 of (n - 1 - j) Y_j,
// so the cell pass keeps W per cell in FP64 (bt_w_next: set at sub-step 0, added to through sub-step n - 2) and the
// last sub-step's edge pass forms the sum from W (bt_acc_of). This replaces a FP64 read and write per edge and sub-step
// by one per cell and sub-step; each edge's sum still comes from one expression, so both of its cells see the same flux.
__device__ __forceinline__ void bt_w_next(double *__restrict__ W, int i, float y, int j, int n) {
  if (j == 0) W[i] = __dmul_rn((double)(n - 1), (double)y);
  else if (j <= n - 2) W[i] = __fma_rn((double)(n - 1 - j), (double)y, W[i]);
}
__device__ __forceinline__ double bt_acc_of(float tau, float G, double wi, double wj, float rde, int n) {
  const double half = 0.5 * (double)n * (double)(n - 1);
  return (double)tau * __fma_rn(-__dsub_rn(wj, wi), (double)rde, __dmul_rn((double)G, half));
}

// ---- fast loop, grid-wide form (stacks without tiles): deviation variables; the cell pass stores Y = Gc (deta +
// gamma (deta - deta_prev)) in deprev for the edge pass, and adds its share to W. Sub-step 0 forms each cell's row of
// constants for the stage (cw32, 32 bytes: the six slot coefficients sign l_e H_e and c0 = their sum against ubar0,
// all over the cell's area, then Gc), which later sub-steps read as two 16-byte loads. ----
__device__ __forceinline__ void bt_eta_cell(const LayersDev &M, float tau, int j, int n, int i) {
  const GridDev &g = M.g;
  int es[6];
  float c[6];
  slots6(g.cellEdge, i, es);
  float c0, gc;
  float4 *row = reinterpret_cast<float4 *>(M.cw32 + (size_t)i * 8);
  if (j == 0) {
    int sg[6];
    signs6(g.cellSign, i, sg);
    const float rA = g.rA32[i];
    c0 = 0.f;
#pragma unroll
    for (int s = 0; s < 6; s++) {
      const int e = es[s];
      const float cs = e >= 0 ? (float)sg[s] * g.le32[e] * M.He32[e] : 0.f;
      if (e >= 0) c0 += cs * (float)M.ub0[e];
      c[s] = __fmul_rn(cs, rA);
    }
    c0 = __fmul_rn(c0, rA);
    gc = M.Gc32[i];
    row[0] = make_float4(c[0], c[1], c[2], c[3]);
    row[1] = make_float4(c[4], c[5], c0, gc);
  } else {
    const float4 r0 = row[0], r1 = row[1];
    c[0] = r0.x; c[1] = r0.y; c[2] = r0.z; c[3] = r0.w; c[4] = r1.x; c[5] = r1.y;
    c0 = r1.z;
    gc = r1.w;
  }
  const float d0 = M.deta[i];
  float div = c0;
#pragma unroll
  for (int s = 0; s < 6; s++)
    if (es[s] >= 0) div = __fmaf_rn(c[s], M.dub[es[s]], div);
  const float dn = bt_eta_new(d0, tau, div);
  M.deta[i] = dn;
  const float y = bt_y_new(gc, (float)M.div_damp, dn, d0);
  M.deprev[i] = y;                           // Y, what the edge pass reads
  bt_w_next(M.wsum, i, y, j, n);
}

// sub-step j of edge e; on the last one (j = n - 1) also its sum acc, from W
__device__ __forceinline__ void bt_u_edge(const LayersDev &M, float tau, int j, int n, int e) {
  const float v = M.dub[e];
  const float *Y = M.deprev;
  const int2 ij = M.g.eIJ[e];
  const float2 gr = M.Gr32[e];
  M.dub[e] = bt_u_new(v, tau, gr.x, Y[ij.x], Y[ij.y], gr.y);
  if (j == n - 1) M.acc[e] = bt_acc_of(tau, gr.x, M.wsum[ij.x], M.wsum[ij.y], gr.y, n);
}

// ---- The split sub-step passes over a wide chunk (up to SUB_W items a thread, THREADS apart): each thread issues the
// plain loads of all its items, then their gathers, then computes and stores, so a thread keeps SUB_W items' loads in
// flight and reads the stack's pointers once for all of them. Per item the arithmetic of bt_u_edge / bt_eta_cell. ----
__device__ __forceinline__ void bt_u_edges(const LayersDev &M, float tau, int j, int n, int first, int end) {
  const int2 *__restrict__ eIJ = M.g.eIJ;
  const float2 *__restrict__ Gr = M.Gr32;
  const float *__restrict__ Y = M.deprev;
  float *__restrict__ dub = M.dub;
  float v[SUB_W], gq[SUB_W], rq[SUB_W], ya[SUB_W], yb[SUB_W];
  int ia[SUB_W], ib[SUB_W];
#pragma unroll
  for (int q = 0; q < SUB_W; q++) {
    const int e = first + q * THREADS;
    v[q] = gq[q] = rq[q] = 0.f;
    ia[q] = ib[q] = 0;
    if (e < end) {
      v[q] = dub[e];
      const float2 gr = Gr[e];
      gq[q] = gr.x;
      rq[q] = gr.y;
      const int2 ij = eIJ[e];
      ia[q] = ij.x;
      ib[q] = ij.y;
    }
  }
#pragma unroll
  for (int q = 0; q < SUB_W; q++) {
    ya[q] = yb[q] = 0.f;
    if (first + q * THREADS < end) {
      ya[q] = Y[ia[q]];
      yb[q] = Y[ib[q]];
    }
  }
#pragma unroll
  for (int q = 0; q < SUB_W; q++) {
    const int e = first + q * THREADS;
    if (e < end) dub[e] = bt_u_new(v[q], tau, gq[q], ya[q], yb[q], rq[q]);
  }
  if (j == n - 1) {
    const double *__restrict__ W = M.wsum;
    double *__restrict__ acc = M.acc;
    double wa[SUB_W], wb[SUB_W];
#pragma unroll
    for (int q = 0; q < SUB_W; q++) {
      wa[q] = wb[q] = 0.0;
      if (first + q * THREADS < end) {
        wa[q] = W[ia[q]];
        wb[q] = W[ib[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < SUB_W; q++) {
      const int e = first + q * THREADS;
      if (e < end) acc[e] = bt_acc_of(tau, gq[q], wa[q], wb[q], rq[q], n);
    }
  }
}

// sub-steps j >= 1 of the cell pass (the slot coefficients and c0 formed by sub-step 0)
template <int W>
__device__ __forceinline__ void bt_eta_cells(const LayersDev &M, float tau, int j, int n, int first, int end) {
  const int *__restrict__ cellEdge = M.g.cellEdge;
  const float4 *__restrict__ rows = reinterpret_cast<const float4 *>(M.cw32);
  const float *__restrict__ dub = M.dub;
  float *__restrict__ deta = M.deta;
  float *__restrict__ Y = M.deprev;
  double *__restrict__ wsum = M.wsum;
  const float gam = (float)M.div_damp;
  for (int base = first; base < end; base += W * THREADS) {
    int es[W][6];
    float c[W][6], u[W][6], cz[W], d0[W], gc[W];
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int i = base + q * THREADS;
      cz[q] = d0[q] = gc[q] = 0.f;
#pragma unroll
      for (int s = 0; s < 6; s++) { es[q][s] = -1; c[q][s] = 0.f; }
      if (i < end) {
        slots6(cellEdge, i, es[q]);
        const float4 r0 = rows[2 * (size_t)i], r1 = rows[2 * (size_t)i + 1];
        c[q][0] = r0.x; c[q][1] = r0.y; c[q][2] = r0.z; c[q][3] = r0.w; c[q][4] = r1.x; c[q][5] = r1.y;
        cz[q] = r1.z;
        gc[q] = r1.w;
        d0[q] = deta[i];
      }
    }
#pragma unroll
    for (int q = 0; q < W; q++)
#pragma unroll
      for (int s = 0; s < 6; s++) u[q][s] = es[q][s] >= 0 ? dub[es[q][s]] : 0.f;
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int i = base + q * THREADS;
      if (i < end) {
        float div = cz[q];
#pragma unroll
        for (int s = 0; s < 6; s++)
          if (es[q][s] >= 0) div = __fmaf_rn(c[q][s], u[q][s], div);
        const float dn = bt_eta_new(d0[q], tau, div);
        deta[i] = dn;
        const float y = bt_y_new(gc[q], gam, dn, d0[q]);
        Y[i] = y;
        bt_w_next(wsum, i, y, j, n);
      }
    }
  }
}

// The layer fluxes of edge e in the last grid-wide sub-step of a batch with no tiled stack, every layer: F (FP64,
// summed by scale_sum_cell) and its FP32 copy (the limited flux of phase D), acc the sub-steps' FP64 sum; the same
// values scale_cell forms
__device__ __forceinline__ void flux_edge(const LayersDev &M, const MStageArgs &a, double acc, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  const float ubs = M.ubs32[e];
  const double ubm = M.ub0[e] + acc * a.inv_n;
  for (int k = 0; k < M.L; k++) {
    const double he = 0.5 * (a.hs[(size_t)k * N + ea] + a.hs[(size_t)k * N + eb]);
    const double F = he * ((double)(a.us[(size_t)k * E + e] - ubs) + ubm);
    M.F[(size_t)k * E + e] = F;
    M.F32[(size_t)k * E + e] = (float)F;
  }
}

// phase C from the fluxes flux_edge stored: the same sums as scale_cell
template <int L>
__device__ __forceinline__ void scale_sum_cell(const LayersDev &M, const MStageArgs &a, int i) {
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
      const double f = M.F[(size_t)k * E + e] * le * a.cdt;
      if (mine) { if (f > 0) out[k] += f; }
      else if (!(f > 0)) out[k] -= f;
    }
  }
  const double A = g.areaCell[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double avail = a.h0[(size_t)k * N + i] - M.floor_;
    const double cap = (avail > 0 ? avail : 0.0) * A;
    M.scale32[(size_t)k * N + i] = out[k] > cap ? __double2float_rz(cap / out[k]) : 1.f;   // rounded toward zero
  }
}

// ---- stage phase C: layer fluxes (FP64) and the floor limiter ----
template <int L>
__device__ __forceinline__ void scale_cell(const LayersDev &M, const MStageArgs &a, int i) {
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
    const int ea = g.eI[e], eb = g.eJ[e];
    const bool mine = ea == i;
    const float ubs = M.ubs32[e];
    const double ubm = M.ub0[e] + M.acc[e] * a.inv_n, le = g.le[e];
#pragma unroll
    for (int k = 0; k < L; k++) {
      const double he = 0.5 * (a.hs[(size_t)k * N + ea] + a.hs[(size_t)k * N + eb]);
      const double F = he * ((double)(a.us[(size_t)k * E + e] - ubs) + ubm);
      if (mine) M.F32[(size_t)k * E + e] = (float)F;
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
    M.scale32[(size_t)k * N + i] = out[k] > cap ? __double2float_rz(cap / out[k]) : 1.f;   // rounded toward zero
  }
}

// ---- stage phase D: h (FP64) and the stage wind ----
// The limited flux of layer k at edge e: the FP32 flux times its upwind cell's FP32 limiter factor, product in FP64.
// One value per edge, used by both cells and by Fm, so volume and tracer mass move between cells exactly.
__device__ __forceinline__ double limited(const LayersDev &M, int k, int e) {
  const GridDev &g = M.g;
  const float f = M.F32[(size_t)k * g.E + e];
  const float sc = f > 0.f ? M.scale32[(size_t)k * g.N + g.eI[e]] : M.scale32[(size_t)k * g.N + g.eJ[e]];
  return (double)f * (double)sc;
}

template <int L>
__device__ __forceinline__ void h_cell(const LayersDev &M, const MStageArgs &a, int i) {
  const GridDev &g = M.g;
  const int N = g.N;
  double div[L];
#pragma unroll
  for (int k = 0; k < L; k++) div[k] = 0;
  int es[6];
  slots6(g.cellEdge, i, es);
  int sg[6];
  signs6(g.cellSign, i, sg);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    if (e < 0) continue;
    const double c = (double)sg[s] * g.le[e];
#pragma unroll
    for (int k = 0; k < L; k++) div[k] += c * limited(M, k, e);
  }
  const double rA = g.rA[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * N + i;
    a.hn[o] = a.h0[o] - a.cdt * div[k] * rA;
  }
}

template <int L>
__device__ __forceinline__ void u_edge(const LayersDev &M, const MStageArgs &a, int e) {
  const GridDev &g = M.g;
  const int E = g.E;
  const float dub = M.dub[e];
  const double le = g.le[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * E + e;
    const float tp = M.Tp32[o];
    if (a.un) {
      if (a.Fm) a.Fm[o] = limited(M, k, e) * le * a.dt;
      a.un[o] = a.u0[o] + (a.cdt * (double)tp + (double)dub);
    } else {
      a.unf[o] = a.u0f[o] + ((float)a.cdt * tp + dub);
    }
  }
}

}  // namespace mixed
}  // namespace isw
