// Phase functions of the time-split RK3 step, plain FP64 form: one call per cell, edge or vertex, every layer of the
// column in one thread. The arithmetic of each phase is the reference kernel's, operation for operation and in the
// same summation order (compiled with -fmad=false), so results are bit-identical to the reference's FP64 path. A cell's
// six slots are walked fully unrolled with a guard on padded slots instead of an early exit, so the gathers of all its
// edges can be in flight together; pads only trail, so each sum keeps the reference's order.
//
// Phase plan of one step (reference layers.py:185-212 with _stage :129-183, Boussinesq branch):
//   init     cells: eta0 = b + sum h (layers.cu:33-38)          edges: ubar0 (layers.cu:64-74)
//   lap x2   cells+vertices: D, zeta (trisk.cu:14-37)          edges: dD/dn - dzeta/dt (trisk.cu:39-45)
//   per stage c = 1/3, 1/2, 1:
//     A      cells: B_k (layers.cu:83-109), eta = eta0          vertices: q_k (fused.cu:82-98)
//     E      edges: h_e, packed (h_e, u, q_e) (layers.cu:254-263), ubar = ubar0, acc = 0
//     S      edges: slow tendency (layers.cu:269-359)
//     n x    cells: eta step (layers.cu:366-377)   then   edges: ubar step (layers.cu:379-388)
//     C      cells: layer fluxes F (layers.cu:392-397, recomputed here per cell edge; the edge's eI cell stores it)
//                   and the floor limiter's scale (layers.cu:401-416)
//     D      cells: h_n with the limited flux (layers.cu:418-441)   edges: Fm, u_n (layers.cu:418-426, :443-447)
//   vmix     edges: interfacial stress (layers.cu:575-593)
#pragma once
#include "common.cuh"

namespace isw {
namespace fp64 {

__device__ __forceinline__ double edge_h(double a, double b) { return 0.5 * (a + b); }

// A layer's thickness at an edge with the shelf option (reference layers.cu:41-45, 59-61): the mean of its two cells,
// or the thinner where the shelf has squeezed one side below `shelf` (only layers flagged on the bed when ob is kept).
__device__ __forceinline__ double shelf_at(const LayersDev &M, int k, int i, int j) {
  const int N = M.g.N;
  return !M.ob || M.ob[(size_t)k * N + i] > 0 || M.ob[(size_t)k * N + j] > 0 ? M.shelf : 0.0;
}

template <bool OPT>
__device__ __forceinline__ double edge_hk(const LayersDev &M, int k, int i, int j, double a, double b) {
  if (OPT && M.shelf > 0) {
    const double sh = shelf_at(M, k, i, j);
    const double m = a < b ? a : b;
    if (sh > 0 && m < sh) return m;
  }
  return 0.5 * (a + b);
}

template <bool OPT>
__device__ __forceinline__ bool walled(const LayersDev &M, int e) { return OPT && M.wall && M.wall[e] == 0; }

// the squeezed-layer flags ob (reference lay_onbed, layers.cu:51-58)
template <int L>
__device__ __forceinline__ void onbed_cell(const LayersDev &M, const double *__restrict__ h, int i) {
  const int N = M.g.N;
  double below = 0;
#pragma unroll
  for (int k = L - 1; k >= 0; k--) {
    const bool stack = k + 1 < L && h[(size_t)k * N + i] < 2 * M.floor_ && h[(size_t)(k + 1) * N + i] < 2 * M.floor_;
    M.ob[(size_t)k * N + i] = below <= (L - 1 - k) * 2 * M.floor_ || stack ? 1.0 : 0.0;
    below += h[(size_t)k * N + i];
  }
}

// ---- init ----
template <int L>
__device__ __forceinline__ void eta0_cell(const LayersDev &M, const double *__restrict__ h, int i) {
  const int N = M.g.N;
  double z = M.b[i];
#pragma unroll
  for (int k = L - 1; k >= 0; k--) z += h[(size_t)k * N + i];
  M.eta0[i] = z;
}

template <int L, bool OPT = true>
__device__ __forceinline__ void ubar0_edge(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u, int e) {
  const int N = M.g.N, E = M.g.E;
  const int a = M.g.eI[e], b = M.g.eJ[e];
  double H = 0, U = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double he = edge_hk<OPT>(M, k, a, b, h[(size_t)k * N + a], h[(size_t)k * N + b]);
    H += he;
    U += he * u[(size_t)k * E + e];
  }
  M.ub0[e] = walled<OPT>(M, e) ? 0.0 : U / H;
}

// ---- vector Laplacian ----
template <int L>
__device__ __forceinline__ void div_cell(const LayersDev &M, const double *__restrict__ u, int i) {
  const GridDev &g = M.g;
  int es[6];
  double c[6];
  slots6(g.cellEdge, i, es);
  int sg[6];
  signs6(g.cellSign, i, sg);
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    c[s] = e >= 0 ? (double)sg[s] * g.le[e] : 0.0;
  }
  const double A = g.areaCell[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *ul = u + (size_t)k * g.E;
    double s = 0;
#pragma unroll
    for (int t = 0; t < 6; t++)
      if (es[t] >= 0) s += c[t] * ul[es[t]];
    M.D1[(size_t)k * g.N + i] = s / A;
  }
}

template <int L>
__device__ __forceinline__ void curl_vertex(const LayersDev &M, const double *__restrict__ u, int v) {
  const GridDev &g = M.g;
  int es[3];
  double c[3];
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const int e = g.vEdge[v * 3 + s];
    es[s] = e;
    c[s] = (double)g.vEdgeSign[v * 3 + s] * g.de[e];
  }
  const double A = g.areaV[v];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *ul = u + (size_t)k * g.E;
    double z = 0;
#pragma unroll
    for (int s = 0; s < 3; s++) z += c[s] * ul[es[s]];
    M.Z1[(size_t)k * g.NV + v] = z / A;
  }
}

template <int L>
__device__ __forceinline__ void lap_edge(const LayersDev &M, double *__restrict__ out, int e) {
  const GridDev &g = M.g;
  const int a = g.eI[e], b = g.eJ[e], v1 = g.ev1[e], v2 = g.ev2[e];
  const double de = g.de[e], le = g.le[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *Dl = M.D1 + (size_t)k * g.N;
    const double *Zl = M.Z1 + (size_t)k * g.NV;
    out[(size_t)k * g.E + e] = (Dl[b] - Dl[a]) / de - (Zl[v2] - Zl[v1]) / le;
  }
}

// ---- stage phase A ----
template <int L, bool OPT = true>
__device__ __forceinline__ void bern_cell(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u, int i) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  double z[L];
  double s = M.b[i];
#pragma unroll
  for (int k = L - 1; k >= 0; k--) { s += h[(size_t)k * N + i]; z[k] = s; }
  int es[6];
  double c[6];
  slots6(g.cellEdge, i, es);
#pragma unroll
  for (int t = 0; t < 6; t++) {
    const int e = es[t];
    c[t] = e >= 0 ? g.le[e] * g.de[e] * 0.25 : 0.0;
  }
  const double A = g.areaCell[i];
  double Mp = 0, P = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    if (OPT && M.sig) {            // per-cell buoyancy (reference layers.cu:90-95): M_k = P_k + sigma_k z_k
      const double sk = M.sig[(size_t)k * N + i], hk = h[(size_t)k * N + i];
      Mp = P + sk * z[k];
      P += sk * hk;
      M.zm[(size_t)k * N + i] = z[k] - 0.5 * hk;
    } else if (k > 0) {
      Mp += M.gp[k - 1] * z[k];
    }
    const double *ul = u + (size_t)k * E;
    double ke = 0;
#pragma unroll
    for (int t = 0; t < 6; t++)
      if (es[t] >= 0) {
        const double ue = ul[es[t]];
        ke += c[t] * ue * ue;
      }
    double Bk = Mp + ke / A;
    if (OPT && M.tide) Bk -= M.tide[i];   // the tide-generating potential (reference layers.cu:106)
    M.B[(size_t)k * N + i] = Bk;
  }
  M.eta[i] = M.eta0[i];
}

template <int L>
__device__ __forceinline__ void pv_vertex(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u, int v) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E, NV = g.NV;
  int cs[3], es[3];
  double kw[3], c[3];
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const int cc = g.vCell[v * 3 + s];
    cs[s] = cc;
    kw[s] = g.kite[cc * 6 + g.vSlot[v * 3 + s]];
    const int e = g.vEdge[v * 3 + s];
    es[s] = e;
    c[s] = (double)g.vEdgeSign[v * 3 + s] * g.de[e];
  }
  const double Av = g.areaV[v], f = M.fV[v];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double *hl = h + (size_t)k * N;
    const double *ul = u + (size_t)k * E;
    double hv = 0, z = 0;
#pragma unroll
    for (int s = 0; s < 3; s++) hv += kw[s] * hl[cs[s]] * 1.0;
#pragma unroll
    for (int s = 0; s < 3; s++) z += c[s] * ul[es[s]];
    M.q[(size_t)k * NV + v] = (z / Av + f) / (hv / Av);
  }
}

// ---- stage phase E ----
template <int L, bool OPT = true>
__device__ __forceinline__ void edge_hq(const LayersDev &M, const double *__restrict__ h, const double *__restrict__ u, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E, NV = g.NV;
  const int a = g.eI[e], b = g.eJ[e], v1 = g.ev1[e], v2 = g.ev2[e];
  constexpr int PS = pk_stride(L);
  double r[PS];
  r[PS - 1] = 0.0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * E + e;
    const double hv = edge_hk<OPT>(M, k, a, b, h[(size_t)k * N + a], h[(size_t)k * N + b]);
    const double qv = 0.5 * (M.q[(size_t)k * NV + v1] + M.q[(size_t)k * NV + v2]);
    M.hedge[o] = hv;
    r[k * 3 + 0] = hv;
    r[k * 3 + 1] = u[o];
    r[k * 3 + 2] = qv;
  }
  double2 *pp = reinterpret_cast<double2 *>(M.pk + (size_t)e * PS);
#pragma unroll
  for (int q = 0; q < PS / 2; q++) pp[q] = make_double2(r[2 * q], r[2 * q + 1]);
  M.ub[e] = M.ub0[e];
  M.acc[e] = 0.0;
}

// ---- stage phase S: slow tendencies ----

// Copy into shared memory the packed records of the distinct edges named by the rows of edge block c (sList), as
// 16-byte pairs: every thread of the block takes part; the caller synchronises before reading.
template <int L>
__device__ __forceinline__ void stage_pk(const LayersDev &M, int c, double *stg) {
  constexpr int PS = pk_stride(L), P2 = PS / 2;
  const int b0 = M.g.sOff[c], n2 = (M.g.sOff[c + 1] - b0) * P2;
  double2 *dst = reinterpret_cast<double2 *>(stg);
  for (int q = threadIdx.x; q < n2; q += blockDim.x) {
    const int r = q / P2;
    dst[q] = reinterpret_cast<const double2 *>(M.pk + (size_t)M.g.sList[b0 + r] * PS)[q - r * P2];
  }
}
// STG: the neighbours' packed records come from `stg`, this block's staged copy of the distinct records its edges'
// rows name (stage_pk), instead of from M.pk; the same values in the same order.
template <int L, bool OPT = true, bool STG = false>
__device__ __forceinline__ void slow_edge(const LayersDev &M, const double *__restrict__ u, double dts, int e,
                                          const double *__restrict__ theta = nullptr, const double *stg = nullptr) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  double he[L], cap[L], qf[L], Q[L];
  constexpr int PS = pk_stride(L);
  const double *pe = M.pk + (size_t)e * PS;
#pragma unroll
  for (int k = 0; k < L; k++) {
    he[k] = M.hedge[(size_t)k * E + e];
    cap[k] = M.thin * he[k];
    qf[k] = pe[k * 3 + 2];
    Q[k] = 0;
  }
  // the row's neighbour ids and weights first (at most EOE_MAX, validated with the grid), then the gathers, all in
  // flight together; the sum runs in row order as the reference's loop does
  const int cnt = g.eoeStart[e + 1] - g.eoeStart[e];
  int ix[EOE_MAX];
  double wv[EOE_MAX];
  if (STG) {
    trisk_loc(g, e, ix);
    trisk_weights(g, e, wv);
  } else {
    trisk_row(g, e, ix, wv);
  }
#pragma unroll
  for (int t = 0; t < EOE_MAX; t++) {
    if (t < cnt) {
      const double wm = wv[t];
      const double2 *pp = reinterpret_cast<const double2 *>((STG ? stg : M.pk) + (size_t)ix[t] * PS);
      double r[PS];
#pragma unroll
      for (int q = 0; q < PS / 2; q++) {
        const double2 v = pp[q];
        r[2 * q] = v.x;
        r[2 * q + 1] = v.y;
      }
#pragma unroll
      for (int k = 0; k < L; k++) {
        double h2 = r[k * 3 + 0];
        if (h2 > cap[k]) h2 = cap[k];
        const double F2 = h2 * r[k * 3 + 1];
        Q[k] += wm * F2 * 0.5 * (qf[k] + r[k * 3 + 2]);
      }
    }
  }
  const int a = g.eI[e], b = g.eJ[e];
  const double de = g.de[e];
  double T[L], sqk[L];
  double H = 0, U = 0, GT = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double ue = u[(size_t)k * E + e];
    const double *Bl = M.B + (size_t)k * N;
    // a layer squeezed by the shelf fades its pressure force and takes a day's drag (reference layers.cu:293-297);
    // shelf off: sq = 1, the force is -(B_J - B_I) / d and the drag term (1 - 1) / 21600 = 0
    const double shk = OPT && M.shelf > 0 ? shelf_at(M, k, a, b) : 0.0;
    const double sq0 = shk > 0 && he[k] < shk ? (he[k] - 2 * M.floor_ > 0 ? (he[k] - 2 * M.floor_) / (shk - 2 * M.floor_) : 0.0) : 1.0;
    const double sq = theta ? 1.0 : sq0;
    sqk[k] = sq0;
    double d = Q[k] - (sq * (Bl[b] - Bl[a])) / de - (M.drag[k] + (1 - sq) / 21600.0) * ue;
    double ck = M.stress[k];
    if (OPT && k == L - 1 && (M.cd_bot > 0 || M.cbot)) {
      // the bottom layer's quadratic stress cd |u| (|u| from the normal and the TRiSK tangential wind) and the internal
      // tide's drag (reference layers.cu:303-311)
      if (M.cd_bot > 0) {
        double vt = 0;
        for (int t = 0; t < cnt; t++) vt += wv[t] * (STG ? stg : M.pk)[(size_t)ix[t] * PS + k * 3 + 1];
        ck += M.cd_bot * sqrt(ue * ue + vt * vt);
      }
      if (M.cbot) ck += M.cbot[e];
    }
    if (ck != 0) {
      const double r = ck / (he[k] > M.floor_ ? he[k] : M.floor_);
      d = d - ((r * dts > 1e-8) ? (1 - exp(-r * dts)) / dts : r) * ue;
    }
    if (theta) {                   // air layers: + pibar grad(theta) (reference layers.cu:322-326)
      const double *tl = theta + (size_t)k * N;
      const double *pl = M.pibar + (size_t)k * N;
      d = d + (0.5 * (pl[a] + pl[b]) * (tl[b] - tl[a])) / de;
    }
    if (OPT && M.sig) {            // per-cell buoyancy: + zm grad(sigma) (reference layers.cu:327-331)
      const double *sl = M.sig + (size_t)k * N;
      const double *zl = M.zm + (size_t)k * N;
      d = d + sq * ((0.5 * (zl[a] + zl[b]) * (sl[b] - sl[a])) / de);
    }
    if (M.nu4 != 0) d = d - M.nu4 * M.L2[(size_t)k * E + e];
    T[k] = d;
    H += he[k];
    U += he[k] * ue;
  }
  if (OPT && theta && M.shelf > 0) {   // air squeezed against the ground takes its neighbours' tendency (layers.cu:341-355)
    double Tn[L];
#pragma unroll
    for (int k = 0; k < L; k++) {
      Tn[k] = T[k];
      if (sqk[k] >= 1) continue;
      double w = 0, s = 0;
      for (int j = k - 1; j >= 0; j--)
        if (sqk[j] >= 1) { w += he[j]; s += he[j] * T[j]; break; }
      for (int j = k + 1; j < L; j++)
        if (sqk[j] >= 1) { w += he[j]; s += he[j] * T[j]; break; }
      if (w > 0) Tn[k] = sqk[k] * T[k] + (1 - sqk[k]) * s / w;
    }
#pragma unroll
    for (int k = 0; k < L; k++) T[k] = Tn[k];
  }
#pragma unroll
  for (int k = 0; k < L; k++) GT += he[k] * T[k];
  const double gm = GT / H;
#pragma unroll
  for (int k = 0; k < L; k++) M.Tp[(size_t)k * E + e] = T[k] - gm;
  M.G[e] = gm;
  M.He[e] = H;
  M.ubs[e] = U / H;
}

// ---- fast mode ----
__device__ __forceinline__ void bt_eta_cell(const LayersDev &M, double tau, int i) {
  const GridDev &g = M.g;
  const double e0 = M.eta[i];
  M.eta_prev[i] = e0;
  int es[6];
  slots6(g.cellEdge, i, es);
  int sg[6];
  signs6(g.cellSign, i, sg);
  double div = 0;
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    if (e >= 0) div += (double)sg[s] * g.le[e] * M.He[e] * M.ub[e];
  }
  M.eta[i] = e0 - (tau * div) / g.areaCell[i];
}

__device__ __forceinline__ void bt_u_edge(const LayersDev &M, double tau, int e) {
  const GridDev &g = M.g;
  const double v = M.ub[e];
  M.acc[e] += v;
  const int i = g.eI[e], j = g.eJ[e];
  const double gam = M.div_damp;
  const double ej = M.Gc[j] * (M.eta[j] + gam * (M.eta[j] - M.eta_prev[j]));
  const double ei = M.Gc[i] * (M.eta[i] + gam * (M.eta[i] - M.eta_prev[i]));
  M.ub[e] = v + tau * ((-(ej - ei)) / g.de[e] + M.G[e]);
  if (walled<true>(M, e)) {        // walls (reference layers.py:173-174)
    M.ub[e] = 0.0;
    M.acc[e] = 0.0;
  }
}


// The batched step's grid-wide form of the two sub-step passes: the cell pass also stores Y = Gc (eta + gamma (eta -
// eta_prev)) (in eta_prev's place), the expression bt_u_edge evaluates for each of an edge's two cells, so the edge
// pass reads two values per edge. Same operations, same bits as bt_eta_cell / bt_u_edge.
__device__ __forceinline__ void bt_eta_cell_y(const LayersDev &M, double tau, int j, int i) {
  const GridDev &g = M.g;
  const double e0 = M.eta[i];
  int es[6];
  slots6(g.cellEdge, i, es);
  // the slot coefficients sign l_e H_e are constant over the stage's sub-steps: formed by sub-step 0, then read back
  // (48-byte rows: three 16-byte loads)
  double c[6];
  if (j == 0) {
    int sg[6];
    signs6(g.cellSign, i, sg);
#pragma unroll
    for (int s = 0; s < 6; s++) {
      const int e = es[s];
      c[s] = e >= 0 ? (double)sg[s] * g.le[e] * M.He[e] : 0.0;
      M.cw[(size_t)i * 6 + s] = c[s];
    }
  } else {
    const double2 *cw = reinterpret_cast<const double2 *>(M.cw + (size_t)i * 6);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const double2 v = cw[q];
      c[2 * q] = v.x;
      c[2 * q + 1] = v.y;
    }
  }
  double div = 0;
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int e = es[s];
    if (e >= 0) div += c[s] * M.ub[e];
  }
  const double en = e0 - (tau * div) / g.areaCell[i];
  M.eta[i] = en;
  M.eta_prev[i] = M.Gc[i] * (en + M.div_damp * (en - e0));
}

template <bool OPT = false>
__device__ __forceinline__ void bt_u_edge_y(const LayersDev &M, double tau, int e) {
  const GridDev &g = M.g;
  const double v = M.ub[e];
  M.acc[e] += v;
  const double *Y = M.eta_prev;
  M.ub[e] = v + tau * ((-(Y[g.eJ[e]] - Y[g.eI[e]])) / g.de[e] + M.G[e]);
  if (walled<OPT>(M, e)) {         // walls (reference layers.py:173-174), as bt_u_edge
    M.ub[e] = 0.0;
    M.acc[e] = 0.0;
  }
}

// ---- The split sub-step passes over a wide chunk (W items a thread, THREADS apart; mixed::bt_u_edges' scheme): the
// plain loads of all the thread's items, then their gathers, then the arithmetic and stores of bt_u_edge_y /
// bt_eta_cell_y (the latter for sub-steps j >= 1). ----
template <int W, bool OPT>
__device__ __forceinline__ void bt_u_edges_y(const LayersDev &M, double tau, int first, int end) {
  const int *__restrict__ eI = M.g.eI;
  const int *__restrict__ eJ = M.g.eJ;
  const double *__restrict__ de = M.g.de;
  const double *__restrict__ G = M.G;
  const double *__restrict__ Y = M.eta_prev;
  double *__restrict__ ub = M.ub;
  double *__restrict__ acc = M.acc;
  for (int base = first; base < end; base += W * THREADS) {
    double v[W], aq[W], gq[W], dq[W], ya[W], yb[W];
    int ia[W], ib[W];
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int e = base + q * THREADS;
      v[q] = aq[q] = gq[q] = 0.0;
      dq[q] = 1.0;
      ia[q] = ib[q] = 0;
      if (e < end) {
        v[q] = ub[e];
        aq[q] = acc[e];
        gq[q] = G[e];
        dq[q] = de[e];
        ia[q] = eI[e];
        ib[q] = eJ[e];
      }
    }
#pragma unroll
    for (int q = 0; q < W; q++) {
      ya[q] = yb[q] = 0.0;
      if (base + q * THREADS < end) {
        ya[q] = Y[ia[q]];
        yb[q] = Y[ib[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int e = base + q * THREADS;
      if (e < end) {
        const bool w = walled<OPT>(M, e);
        acc[e] = w ? 0.0 : aq[q] + v[q];
        ub[e] = w ? 0.0 : v[q] + tau * ((-(yb[q] - ya[q])) / dq[q] + gq[q]);
      }
    }
  }
}

template <int W>
__device__ __forceinline__ void bt_eta_cells_y(const LayersDev &M, double tau, int first, int end) {
  const int *__restrict__ cellEdge = M.g.cellEdge;
  const double *__restrict__ cwt = M.cw;
  const double *__restrict__ area = M.g.areaCell;
  const double *__restrict__ Gc = M.Gc;
  const double *__restrict__ ub = M.ub;
  double *__restrict__ eta = M.eta;
  double *__restrict__ Y = M.eta_prev;
  const double gam = M.div_damp;
  for (int base = first; base < end; base += W * THREADS) {
    int es[W][6];
    double c[W][6], u[W][6], e0[W], ar[W], gc[W];
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int i = base + q * THREADS;
      e0[q] = gc[q] = 0.0;
      ar[q] = 1.0;
#pragma unroll
      for (int s = 0; s < 6; s++) { es[q][s] = -1; c[q][s] = 0.0; }
      if (i < end) {
        slots6(cellEdge, i, es[q]);
        const double2 *cw = reinterpret_cast<const double2 *>(cwt + (size_t)i * 6);
#pragma unroll
        for (int h = 0; h < 3; h++) {
          const double2 x = cw[h];
          c[q][2 * h] = x.x;
          c[q][2 * h + 1] = x.y;
        }
        e0[q] = eta[i];
        ar[q] = area[i];
        gc[q] = Gc[i];
      }
    }
#pragma unroll
    for (int q = 0; q < W; q++)
#pragma unroll
      for (int s = 0; s < 6; s++) u[q][s] = es[q][s] >= 0 ? ub[es[q][s]] : 0.0;
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int i = base + q * THREADS;
      if (i < end) {
        double div = 0;
#pragma unroll
        for (int s = 0; s < 6; s++)
          if (es[q][s] >= 0) div += c[q][s] * u[q][s];
        const double en = e0[q] - (tau * div) / ar[q];
        eta[i] = en;
        Y[i] = gc[q] * (en + gam * (en - e0[q]));
      }
    }
  }
}

// The layer fluxes of edge e once the stage's fast loop has finished (reference lay_flux, layers.cu:392-397), every
// layer: F = h_e (u - ubar_s) + h_e acc / n, acc the sub-steps' sum of ubar. A batch with no tiled stack forms them in
// the last grid-wide sub-step's edge pass, once per edge, and its phase C only sums them (scale_sum_cell); batches
// with tiles recompute them in phase C (scale_cell: the tile kernel's tail has no spare parallelism for the gathers).
template <bool OPT = true>
__device__ __forceinline__ void flux_edge(const LayersDev &M, const StageArgs &a, double acc, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const int ea = g.eI[e], eb = g.eJ[e];
  const double ubs = M.ubs[e];
  for (int k = 0; k < M.L; k++) {
    const double he = edge_hk<OPT>(M, k, ea, eb, a.hs[(size_t)k * N + ea], a.hs[(size_t)k * N + eb]);
    M.F[(size_t)k * E + e] = walled<OPT>(M, e) ? 0.0 : he * (a.us[(size_t)k * E + e] - ubs) + he * (acc * a.inv_n);
  }
}

// phase C from the fluxes flux_edge stored: the same sums as scale_cell
template <int L>
__device__ __forceinline__ void scale_sum_cell(const LayersDev &M, const StageArgs &a, int i) {
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
    M.scale[(size_t)k * N + i] = out[k] > cap ? cap / out[k] : 1.0;
  }
}

// ---- stage phase C: layer fluxes and the floor limiter's scale ----
template <int L, bool OPT = true>
__device__ __forceinline__ void scale_cell(const LayersDev &M, const StageArgs &a, int i) {
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
    const double ubs = M.ubs[e], acc = M.acc[e], le = g.le[e];
#pragma unroll
    for (int k = 0; k < L; k++) {
      const double he = edge_hk<OPT>(M, k, ea, eb, a.hs[(size_t)k * N + ea], a.hs[(size_t)k * N + eb]);
      const double F = walled<OPT>(M, e) ? 0.0 : he * (a.us[(size_t)k * E + e] - ubs) + he * (acc * a.inv_n);
      if (mine) M.F[(size_t)k * E + e] = F;
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

// ---- stage phase D ----
__device__ __forceinline__ double limited(const LayersDev &M, int k, int e) {
  const GridDev &g = M.g;
  double f = M.F[(size_t)k * g.E + e];
  f *= f > 0 ? M.scale[(size_t)k * g.N + g.eI[e]] : M.scale[(size_t)k * g.N + g.eJ[e]];
  return f;
}

template <int L>
__device__ __forceinline__ void h_cell(const LayersDev &M, const StageArgs &a, int i) {
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
  const double A = g.areaCell[i];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * N + i;
    a.hn[o] = a.h0[o] - (a.cdt * div[k]) / A;
  }
}

template <int L, bool OPT = true>
__device__ __forceinline__ void u_edge(const LayersDev &M, const StageArgs &a, int e) {
  const GridDev &g = M.g;
  const int E = g.E;
  const double dub = M.ub[e] - M.ub0[e];
  const double le = g.le[e];
#pragma unroll
  for (int k = 0; k < L; k++) {
    const size_t o = (size_t)k * E + e;
    if (a.Fm) a.Fm[o] = limited(M, k, e) * le * a.dt;
    a.un[o] = walled<OPT>(M, e) ? 0.0 : a.u0[o] + a.cdt * M.Tp[o] + dub;
  }
}

// ---- after the stages: interfacial stress ----
template <int L, bool OPT = true>
__device__ __forceinline__ void vmix_edge(const LayersDev &M, const double *__restrict__ h, double *__restrict__ u, double dt, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const int ia = g.eI[e], ib = g.eJ[e];
  const double c = M.vmix, cd = M.vmix_cd;
  double d = 0;
#pragma unroll
  for (int k = 0; k + 1 < L; k++) {
    const double ha = 0.5 * (h[(size_t)k * N + ia] + h[(size_t)k * N + ib]);
    const double hb = 0.5 * (h[(size_t)(k + 1) * N + ia] + h[(size_t)(k + 1) * N + ib]);
    double *ua = u + (size_t)k * E + e;
    double *ub = u + (size_t)(k + 1) * E + e;
    const double mean = (ha * *ua + hb * *ub) / (ha + hb);
    const double du0 = *ua - *ub;
    double du1 = du0 * exp(-c * (1 / ha + 1 / hb) * dt);
    if (cd > 0) du1 = du1 / (1 + cd * fabs(du0) * (1 / ha + 1 / hb) * dt);
    *ua = mean + hb / (ha + hb) * du1;
    *ub = mean - ha / (ha + hb) * du1;
    d += 0.5 * ha * hb / (ha + hb) * (du0 * du0 - du1 * du1);
  }
  M.diss[e] = d;
  if (walled<OPT>(M, e))
    for (int k = 0; k < L; k++) u[(size_t)k * E + e] = 0.0;
}

}  // namespace fp64
}  // namespace isw
