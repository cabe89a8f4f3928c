/* CPU oracle: a plain-C restatement of the reference's hot-path kernels, FP64, in the reference's own summation order.
 *
 * TEST INFRASTRUCTURE ONLY. The product never links, loads or calls this file; tests, smoke() and bench.py's CPU-baseline
 * leg use it as the checker (and as the timed "port" baseline).
 *
 * Each function restates one reference kernel (file:line given at each) as a loop over its whole domain. Arguments are
 * the reference kernel's own argument list, preceded by `rows` (the reference's blockIdx.y extent: layers, or tracer x
 * layer rows for transport; 1 for whole-column kernels). Option pointers the reference passes as NULL when an option is
 * off (sig, zm, tide, theta, pibar, ob, cbot) must be NULL here: those branches are not restated, and a non-NULL one
 * sets the error flag (o_error()) and leaves the outputs untouched.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp -shared -fPIC (no fused multiply-add, the host counterpart of the
 * reference's --fmad=false), so every + - * / and sqrt rounds exactly as the reference's FP64 GPU build does; exp()
 * comes from libm and may differ from CUDA's in the last bit.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

typedef double real;
#define LMAX 8

static int g_error = 0;
int o_error(void) { int e = g_error; g_error = 0; return e; }
#define REFUSE(cond) do { if (cond) { g_error = 1; return; } } while (0)

/* edge thickness of a layer: the two cells' mean, or the thinner under the shelf option (reference layers.cu:41-45) */
static inline real edge_h(real a, real b, real shelf) {
  const real m = a < b ? a : b;
  return shelf > 0 && m < shelf ? m : (real)0.5 * (a + b);
}

/* reference layers.cu:33-38 */
void o_lay_eta(int rows, int N, int L, const real* h, const real* b, real* eta) {
  (void)rows;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    real z = b[i];
    for (int k = L - 1; k >= 0; k--) z += h[(size_t)k * N + i];
    eta[i] = z;
  }
}

/* reference layers.cu:64-74 (ob NULL: the shelf applies to every layer) */
void o_lay_ubar(int rows, int N, int E, int L, const real* h, const real* u, const int* eI, const int* eJ, real shelf,
                real* ubar, const real* ob) {
  (void)rows;
  REFUSE(ob != NULL);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < E; e++) {
    real H = 0, U = 0;
    for (int k = 0; k < L; k++) {
      const real he = edge_h(h[(size_t)k * N + eI[e]], h[(size_t)k * N + eJ[e]], shelf);
      H += he;
      U += he * u[(size_t)k * E + e];
    }
    ubar[e] = U / H;
  }
}

/* reference layers.cu:83-109, fixed-g' branch (sig, zm, tide NULL) */
void o_lay_bern(int rows, int N, int E, int L, const real* h, const real* u, const real* b, const real* gp,
                const int* cellEdge, const real* le, const real* de, const real* areaCell, real* B,
                const real* sig, real* zm, const real* tide) {
  (void)rows;
  REFUSE(sig != NULL || zm != NULL || tide != NULL);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    real z[LMAX];
    real s = b[i];
    for (int k = L - 1; k >= 0; k--) { s += h[(size_t)k * N + i]; z[k] = s; }
    real Mp = 0;
    for (int k = 0; k < L; k++) {
      if (k > 0) Mp += gp[k - 1] * z[k];
      const real* ul = u + (size_t)k * E;
      real ke = 0;
      for (int m = 0; m < 6; m++) {
        const int e = cellEdge[i * 6 + m];
        if (e < 0) break;
        ke += le[e] * de[e] * (real)0.25 * ul[e] * ul[e];
      }
      B[(size_t)k * N + i] = Mp + ke / areaCell[i];
    }
  }
}

/* reference fused.cu:82-98 (FP64: DIVBY divides) */
void o_swe_vertex(int rows, int N, int E, int NV, const real* h, const real* u, const int* vCell, const signed char* vSlot,
                  const real* kite, const int* vEdge, const signed char* vEdgeSign, const real* de, const real* areaV,
                  const real* fV, real* q) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int v = 0; v < NV; v++) {
      const real* hl = h + (size_t)l * N;
      const real* ul = u + (size_t)l * E;
      real hv = 0, z = 0;
      for (int k = 0; k < 3; k++) {
        const int c = vCell[v * 3 + k];
        hv += kite[c * 6 + vSlot[v * 3 + k]] * hl[c] * (real)1;
      }
      for (int k = 0; k < 3; k++) {
        const int e = vEdge[v * 3 + k];
        z += (real)vEdgeSign[v * 3 + k] * de[e] * ul[e];
      }
      q[(size_t)l * NV + v] = (z / areaV[v] + fV[v]) / (hv / areaV[v]);
    }
}

/* reference layers.cu:254-263 (pk packed [edge][layer][h_e, u, q_e]; rows = L) */
void o_lay_edge_hq(int rows, int N, int E, int NV, const real* h, const real* q, const int* eI, const int* eJ,
                   const int* ev1, const int* ev2, real shelf, const real* u, real* he, real* pk, const real* ob) {
  REFUSE(ob != NULL);
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int e = 0; e < E; e++) {
      const size_t o = (size_t)l * E + e;
      const real hv = edge_h(h[(size_t)l * N + eI[e]], h[(size_t)l * N + eJ[e]], shelf);
      const real qv = (real)0.5 * (q[(size_t)l * NV + ev1[e]] + q[(size_t)l * NV + ev2[e]]);
      he[o] = hv;
      real* pp = pk + ((size_t)e * rows + l) * 3;
      pp[0] = hv; pp[1] = u[o]; pp[2] = qv;
    }
}

/* reference layers.cu:269-359, Boussinesq branch: theta, pibar, sig, zm, ob, cbot NULL and cd_bot 0 */
void o_lay_slow(int rows, int N, int E, int L, const real* pk, const real* wf, const real* hedge, const real* u, const real* B,
                const int* eoeStart, const int* eoe, const int* eI, const int* eJ, const real* de, const real* drag,
                const real* stress, real floor_, real nu4, const real* lap4, const real* theta, const real* pibar,
                real dts, real thin, real shelf, real* Tp, real* G, real* He, real* ubs, const real* sig, const real* zm,
                const real* ob, real cd_bot, const real* cbot) {
  (void)rows;
  REFUSE(theta != NULL || pibar != NULL || sig != NULL || zm != NULL || ob != NULL || cbot != NULL || cd_bot > 0);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < E; e++) {
    real T[LMAX], hev[LMAX];
    real H = 0, U = 0, GT = 0;
    for (int k = 0; k < L; k++) {
      const real* hl = hedge + (size_t)k * E;
      const real* ul = u + (size_t)k * E;
      const real* Bl = B + (size_t)k * N;
      const real he = hl[e];
      const real cap = thin * he, qf = pk[((size_t)e * L + k) * 3 + 2];
      real Q = 0;
      for (int m = eoeStart[e]; m < eoeStart[e + 1]; m++) {
        const real* pp = pk + ((size_t)eoe[m] * L + k) * 3;
        real h2 = pp[0];
        if (h2 > cap) h2 = cap;
        const real F2 = h2 * pp[1];
        Q += wf[m] * F2 * (real)0.5 * (qf + pp[2]);
      }
      const real shk = shelf;
      const real sq0 = shk > 0 && he < shk ? (he - 2 * floor_ > 0 ? (he - 2 * floor_) / (shk - 2 * floor_) : (real)0) : (real)1;
      const real sq = sq0;
      real d = Q - (sq * (Bl[eJ[e]] - Bl[eI[e]])) / de[e] - (drag[k] + (1 - sq) / (real)21600) * ul[e];
      const real ck = stress[k];
      if (ck != 0) {
        const real r = ck / (he > floor_ ? he : floor_);
        d = d - ((r * dts > (real)1e-8) ? (1 - exp(-r * dts)) / dts : r) * ul[e];
      }
      if (nu4 != 0) d = d - nu4 * lap4[(size_t)k * E + e];
      T[k] = d;
      hev[k] = he;
      H += he;
      U += he * ul[e];
    }
    for (int k = 0; k < L; k++) GT += hev[k] * T[k];
    const real g = GT / H;
    for (int k = 0; k < L; k++) Tp[(size_t)k * E + e] = T[k] - g;
    G[e] = g;
    He[e] = H;
    ubs[e] = U / H;
  }
}

/* reference trisk.cu:14-25 */
void o_cell_div(int rows, int N, int E, const real* u, const int* cellEdge, const signed char* cellSign, const real* le,
                const real* areaCell, real* D) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int i = 0; i < N; i++) {
      const real* ul = u + (size_t)l * E;
      real s = 0;
      for (int k = 0; k < 6; k++) {
        const int e = cellEdge[i * 6 + k];
        if (e < 0) break;
        s += (real)cellSign[i * 6 + k] * le[e] * ul[e];
      }
      D[(size_t)l * N + i] = s / areaCell[i];
    }
}

/* reference trisk.cu:27-37 */
void o_vertex_curl(int rows, int E, int NV, const real* u, const int* vEdge, const signed char* vEdgeSign, const real* de,
                   const real* areaV, real* Z) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int v = 0; v < NV; v++) {
      const real* ul = u + (size_t)l * E;
      real z = 0;
      for (int k = 0; k < 3; k++) {
        const int e = vEdge[v * 3 + k];
        z += (real)vEdgeSign[v * 3 + k] * de[e] * ul[e];
      }
      Z[(size_t)l * NV + v] = z / areaV[v];
    }
}

/* reference trisk.cu:39-45 */
void o_edge_lap(int rows, int N, int E, int NV, const real* D, const real* Z, const int* eI, const int* eJ, const int* ev1,
                const int* ev2, const real* de, const real* le, real* out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int e = 0; e < E; e++) {
      const real* Dl = D + (size_t)l * N;
      const real* Zl = Z + (size_t)l * NV;
      out[(size_t)l * E + e] = (Dl[eJ[e]] - Dl[eI[e]]) / de[e] - (Zl[ev2[e]] - Zl[ev1[e]]) / le[e];
    }
}

/* reference layers.cu:366-377 */
void o_bt_eta(int rows, int N, const real* He, const real* ub, const int* cellEdge, const signed char* cellSign,
              const real* le, const real* areaCell, real tau, real* eta, real* eta_prev) {
  (void)rows;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    eta_prev[i] = eta[i];
    real div = 0;
    for (int m = 0; m < 6; m++) {
      const int e = cellEdge[i * 6 + m];
      if (e < 0) break;
      div += (real)cellSign[i * 6 + m] * le[e] * He[e] * ub[e];
    }
    eta[i] = eta[i] - (tau * div) / areaCell[i];
  }
}

/* reference layers.cu:379-388 */
void o_bt_u(int rows, int E, const real* eta, const real* eta_prev, real gamma, const real* G, const int* eI, const int* eJ,
            const real* de, const real* Gc, real tau, real* ub, real* acc) {
  (void)rows;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < E; e++) {
    const real v = ub[e];
    acc[e] += v;
    const int i = eI[e], j = eJ[e];
    const real ej = Gc[j] * (eta[j] + gamma * (eta[j] - eta_prev[j]));
    const real ei = Gc[i] * (eta[i] + gamma * (eta[i] - eta_prev[i]));
    ub[e] = v + tau * ((-(ej - ei)) / de[e] + G[e]);
  }
}

/* reference layers.cu:392-397 */
void o_lay_flux(int rows, int N, int E, const real* h, const real* u, const real* ubs, const real* acc, real inv_n,
                const int* eI, const int* eJ, real shelf, real* F, const real* ob) {
  REFUSE(ob != NULL);
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int e = 0; e < E; e++) {
      const real he = edge_h(h[(size_t)l * N + eI[e]], h[(size_t)l * N + eJ[e]], shelf);
      F[(size_t)l * E + e] = he * (u[(size_t)l * E + e] - ubs[e]) + he * (acc[e] * inv_n);
    }
}

/* reference layers.cu:401-416 */
void o_lay_scale(int rows, int N, int E, const real* h0, const real* F, const int* cellEdgeAsc, const int* eI, const real* le,
                 const real* areaCell, real dts, real floor_, real* scale) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int i = 0; i < N; i++) {
      const real* Fl = F + (size_t)l * E;
      real out = 0;
      for (int m = 0; m < 6; m++) {
        const int e = cellEdgeAsc[i * 6 + m];
        if (e < 0) break;
        const real f = Fl[e] * le[e] * dts;
        if (eI[e] == i) { if (f > 0) out += f; }
        else if (!(f > 0)) out -= f;
      }
      const real avail = h0[(size_t)l * N + i] - floor_;
      const real cap = (avail > 0 ? avail : (real)0) * areaCell[i];
      scale[(size_t)l * N + i] = out > cap ? cap / out : (real)1;
    }
}

/* reference layers.cu:418-426 */
void o_lay_limit(int rows, int N, int E, const int* eI, const int* eJ, const real* scale, const real* le, real dt, real* F,
                 real* Fm) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int e = 0; e < E; e++) {
      const size_t o = (size_t)l * E + e;
      real f = F[o];
      f *= f > 0 ? scale[(size_t)l * N + eI[e]] : scale[(size_t)l * N + eJ[e]];
      F[o] = f;
      if (Fm) Fm[o] = f * le[e] * dt;
    }
}

/* reference layers.cu:429-441 */
void o_lay_h(int rows, int N, int E, const real* h0, const real* F, const int* cellEdge, const signed char* cellSign,
             const real* le, const real* areaCell, real cdt, real* hn) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int i = 0; i < N; i++) {
      const real* Fl = F + (size_t)l * E;
      real div = 0;
      for (int m = 0; m < 6; m++) {
        const int e = cellEdge[i * 6 + m];
        if (e < 0) break;
        div += (real)cellSign[i * 6 + m] * le[e] * Fl[e];
      }
      const size_t o = (size_t)l * N + i;
      hn[o] = h0[o] - (cdt * div) / areaCell[i];
    }
}

/* reference layers.cu:443-447 */
void o_lay_u(int rows, int E, const real* u0, const real* Tp, const real* ub_end, const real* ub0, real cdt, real* un) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int e = 0; e < E; e++) {
      const size_t o = (size_t)l * E + e;
      un[o] = u0[o] + cdt * Tp[o] + (ub_end[e] - ub0[e]);
    }
}

/* reference layers.cu:575-593: interfacial stress between neighbouring layers, top down */
void o_lay_vmix(int rows, int N, int E, int L, const real* h, const int* eI, const int* eJ, real c, real dt, real* u,
                real* diss, real cd) {
  (void)rows;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < E; e++) {
    real d = 0;
    for (int k = 0; k + 1 < L; k++) {
      const real ha = (real)0.5 * (h[(size_t)k * N + eI[e]] + h[(size_t)k * N + eJ[e]]);
      const real hb = (real)0.5 * (h[(size_t)(k + 1) * N + eI[e]] + h[(size_t)(k + 1) * N + eJ[e]]);
      real* ua = u + (size_t)k * E + e;
      real* ub = u + (size_t)(k + 1) * E + e;
      const real mean = (ha * *ua + hb * *ub) / (ha + hb);
      const real du0 = *ua - *ub;
      real du1 = du0 * exp(-c * (1 / ha + 1 / hb) * dt);
      if (cd > 0) du1 = du1 / (1 + cd * fabs(du0) * (1 / ha + 1 / hb) * dt);
      *ua = mean + hb / (ha + hb) * du1;
      *ub = mean - ha / (ha + hb) * du1;
      d += (real)0.5 * ha * hb / (ha + hb) * (du0 * du0 - du1 * du1);
    }
    diss[e] = d;
  }
}

/* reference trisk.cu:48-59 */
void o_mass_update(int rows, int N, int E, const real* M0, const real* Fm, const int* cellEdgeAsc, const int* eI, real* M1) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int l = 0; l < rows; l++)
    for (int i = 0; i < N; i++) {
      const size_t o = (size_t)l * N + i;
      const real* f = Fm + (size_t)l * E;
      real m = M0[o];
      for (int k = 0; k < 6; k++) {
        const int e = cellEdgeAsc[i * 6 + k];
        if (e < 0) break;
        if (eI[e] == i) m -= f[e]; else m += f[e];
      }
      M1[o] = m;
    }
}

/* ---- FCT transport: rows y = tracer * Lm + layer (reference fused.cu:140-143) ---- */

/* reference fused.cu:124-127 */
static inline real upwind(const real* Fml, const real* p, const int* eI, const int* eJ, int e) {
  const real f = Fml[e];
  return f * (f >= 0 ? p[eI[e]] : p[eJ[e]]);
}

/* reference fused.cu:131-138 (FP64: the stencil field and weights are the 64-bit ones) */
static inline real hoflux(const real* Fml, const real* ps, const real* psf, const int* idx, const real* wt, const int* eI,
                          const int* eJ, int e, real beta) {
  const real f = Fml[e];
  const int o = e * 8;
  const real a = wt[o] * psf[idx[o]] + wt[o + 1] * psf[idx[o + 1]] + wt[o + 2] * psf[idx[o + 2]] + wt[o + 3] * psf[idx[o + 3]];
  const real b = wt[o + 4] * psf[idx[o + 4]] + wt[o + 5] * psf[idx[o + 5]] + wt[o + 6] * psf[idx[o + 6]] + wt[o + 7] * psf[idx[o + 7]];
  return f * ((real)0.5 * (ps[eI[e]] + ps[eJ[e]]) - (real)(a + b)) + fabs(f) * ((real)(b - a) * beta);
}

/* reference fused.cu:146-160 */
void o_tr_td(int rows, int N, int E, int Lm, const real* M0, const real* psi, const real* Fm, const real* M1,
             const int* cellEdgeAsc, const int* eI, const int* eJ, real* td) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int i = 0; i < N; i++) {
      const int l = y % Lm;
      const size_t o = (size_t)y * N + i, om = (size_t)l * N + i;
      const real* p = psi + (size_t)y * N;
      const real* Fml = Fm + (size_t)l * E;
      real t = M0[om] * psi[o];
      for (int k = 0; k < 6; k++) {
        const int e = cellEdgeAsc[i * 6 + k];
        if (e < 0) break;
        const real f = upwind(Fml, p, eI, eJ, e);
        if (eI[e] == i) t -= f; else t += f;
      }
      td[o] = t / M1[om];
    }
}

/* reference fused.cu:163-167 */
void o_tr_hflux(int rows, int E, int Lm, const real* src, const real* srcf, real frac, const real* Fm, const int* idx,
                const real* wt, const int* eI, const int* eJ, int N, real beta, real* Hf) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int e = 0; e < E; e++) {
      const int l = y % Lm;
      Hf[(size_t)y * E + e] = frac * hoflux(Fm + (size_t)l * E, src + (size_t)y * N, srcf + (size_t)y * N, idx, wt, eI, eJ, e, beta);
    }
}

/* reference fused.cu:170-186 */
void o_tr_stage(int rows, int N, int E, int Lm, const real* M0, const real* psi, const real* Hf, real frac, const real* Fm,
                const int* cellEdgeAsc, const int* eI, real* out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int i = 0; i < N; i++) {
      const int l = y % Lm;
      const size_t o = (size_t)y * N + i, om = (size_t)l * N + i;
      const real* Hl = Hf + (size_t)y * E;
      const real* Fml = Fm + (size_t)l * E;
      real t = M0[om] * psi[o];
      real mx = M0[om];
      for (int k = 0; k < 6; k++) {
        const int e = cellEdgeAsc[i * 6 + k];
        if (e < 0) break;
        const real f = Hl[e];
        const real m = frac * Fml[e];
        if (eI[e] == i) { t -= f; mx -= m; } else { t += f; mx += m; }
      }
      out[o] = t / mx;
    }
}

/* reference fused.cu:189-194 */
void o_tr_aflux(int rows, int E, int Lm, const real* psi, const real* p2, const real* p2f, const real* Fm, const int* idx,
                const real* wt, const int* eI, const int* eJ, int N, real beta, real* A) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int e = 0; e < E; e++) {
      const int l = y % Lm;
      const real* Fml = Fm + (size_t)l * E;
      A[(size_t)y * E + e] = hoflux(Fml, p2 + (size_t)y * N, p2f + (size_t)y * N, idx, wt, eI, eJ, e, beta)
                             - upwind(Fml, psi + (size_t)y * N, eI, eJ, e);
    }
}

/* reference fused.cu:197-222 */
void o_tr_ratios(int rows, int N, int E, int Lm, const real* psi, const real* td, const real* M1, const real* A,
                 const int* nbr, const int* cellEdgeAsc, const int* eI, real* Rp, real* Rm) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int i = 0; i < N; i++) {
      const int l = y % Lm;
      const real* p = psi + (size_t)y * N;
      const real* t = td + (size_t)y * N;
      const real* Al = A + (size_t)y * E;
      real hi = fmax(p[i], t[i]), lo = fmin(p[i], t[i]);
      for (int k = 0; k < 6; k++) {
        const int j = nbr[i * 6 + k];
        if (j < 0) break;
        hi = fmax(hi, fmax(p[j], t[j]));
        lo = fmin(lo, fmin(p[j], t[j]));
      }
      const real m1 = M1[(size_t)l * N + i];
      const real qmax = (hi - t[i]) * m1, qmin = (t[i] - lo) * m1;
      real Pp = 0, Pm = 0;
      for (int k = 0; k < 6; k++) {
        const int e = cellEdgeAsc[i * 6 + k];
        if (e < 0) break;
        const real a = Al[e];
        if (eI[e] == i) { if (a > 0) Pm += a; else Pp -= a; }
        else { if (a > 0) Pp += a; else Pm -= a; }
      }
      Rp[(size_t)y * N + i] = Pp > 0 ? fmin((real)1, qmax / Pp) : (real)0;
      Rm[(size_t)y * N + i] = Pm > 0 ? fmin((real)1, qmin / Pm) : (real)0;
    }
}

/* reference fused.cu:225-241 */
void o_tr_apply(int rows, int N, int E, int Lm, const real* td, const real* M1, const real* A, const real* Rp, const real* Rm,
                const int* cellEdgeAsc, const int* eI, const int* eJ, real* psi_out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int y = 0; y < rows; y++)
    for (int i = 0; i < N; i++) {
      const int l = y % Lm;
      const size_t o = (size_t)y * N + i, om = (size_t)l * N + i;
      const real* Al = A + (size_t)y * E;
      const real* rp = Rp + (size_t)y * N;
      const real* rm = Rm + (size_t)y * N;
      real t = td[o] * M1[om];
      for (int k = 0; k < 6; k++) {
        const int e = cellEdgeAsc[i * 6 + k];
        if (e < 0) break;
        const real a = Al[e];
        const real c = a > 0 ? fmin(rp[eJ[e]], rm[eI[e]]) : fmin(rp[eI[e]], rm[eJ[e]]);
        if (eI[e] == i) t -= c * a; else t += c * a;
      }
      psi_out[o] = t / M1[om];
    }
}

/* ---- deterministic sum (reference kernels/trisk.cu:61-81, driven by gpu.py:111-126) ----
 * One pass: block b sums x[b*2048 ...]; thread t adds x[base + t + 256 k] for k = 0..7 in order, then the 256 partials
 * halve pairwise (s[t] += s[t + h], h = 128 .. 1). Passes repeat until one block remains. */
static void block_sum_pass(long long n, const real* x, const real* y, real* out, long long blocks) {
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < blocks; b++) {
    real s[256];
    const long long base = b * 2048;
    for (int t = 0; t < 256; t++) {
      real acc = 0;
      for (int k = 0; k < 8; k++) {
        const long long i = base + t + (long long)k * 256;
        if (i < n) acc += y ? x[i] * y[i] : x[i];
      }
      s[t] = acc;
    }
    for (int h = 128; h > 0; h >>= 1)
      for (int t = 0; t < h; t++) s[t] += s[t + h];
    out[b] = s[0];
  }
}

/* returns the sum; passes ping-pong between two buffers allocated here */
real o_dsum(long long n, const real* x, const real* y) {
  long long blocks = (n + 2047) / 2048;
  real* a = (real*)malloc(sizeof(real) * (size_t)(blocks > 0 ? blocks : 1));
  real* b = (real*)malloc(sizeof(real) * (size_t)((blocks + 2047) / 2048 + 1));
  block_sum_pass(n, x, y, a, blocks);
  while (blocks > 1) {
    const long long m = blocks;
    blocks = (m + 2047) / 2048;
    block_sum_pass(m, a, NULL, b, blocks);
    real* t = a; a = b; b = t;
  }
  const real r = a[0];
  free(a);
  free(b);
  return r;
}
