// Shared definitions of the isw dynamical core: device-side grid and layer descriptors, error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>
#include <vector>

#include "../../include/isw.h"

namespace isw {

constexpr int LMAX = 8;          // layers per column (reference layers.py:30)
constexpr int TRMAX = 16;        // tracers moved in one transport call
constexpr int THREADS = 256;     // threads per block of the phase kernels
// Items per thread of the grid-wide sub-step passes (their chunks hold that many x THREADS): the mixed form's edges,
// the FP64 form's edges, and the cells of both (two a thread raised the cell pass to 75 (mixed) and 100 (FP64)
// registers, and it ran slower at the lower occupancy; FP64 edges ran fastest at two: 8 level-6 members 3.84 ms a
// step against 4.24 at one).
constexpr int SUB_W = 4;
constexpr int SUB_W_FP64 = 2;
constexpr int SUB_WC = 1;
constexpr int EOE_MAX = 10;      // TRiSK row length: the other edges of an edge's two cells (5 + 5 on hexagons)
// The FP64 packed edge record: per edge, (h_e, u, q_e) of each layer, the edge's row padded to an even count of
// doubles so that every row starts on a 16-byte boundary and is read as 16-byte pairs.
__host__ __device__ constexpr int pk_stride(int L) { return (3 * L + 1) & ~1; }

// Thrown inside the library, turned into a status at the C ABI.
struct Error {
  int status;
  std::string msg;
};

void set_last_error(const std::string &m);
[[noreturn]] void fail(int status, const std::string &m);
void check_cuda(cudaError_t e, const char *what);
#define ISW_CUDA(call) ::isw::check_cuda((call), #call)

// The grid on the device: index tables int32 (pads -1), signs and slots int8, geometry FP64, plus FP32 copies of what the
// mixed form reads (weights, stencil weights, reciprocals of the metrics it divides by).
struct GridDev {
  int N, E, NV, nE2;              // nE2 = eoeStart[E], the length of the TRiSK CSR
  const int *eI, *eJ, *nbr, *cellEdge, *cellEdgeAsc, *ev1, *ev2, *vEdge, *vCell, *eoeStart, *eoe, *d2idx;
  const int2 *eIJ;                // (eI, eJ) per edge, one 8-byte load
  const int8_t *cellSign, *vEdgeSign, *vSlot;
  const double *le, *de, *areaCell, *areaV, *fV, *kite, *w, *d2wt;
  const float *w32, *d2wt32, *le32, *de32, *rde32, *rle32, *rA32, *rAV32, *kite32;
  const double *rA, *rde, *rAV;   // FP64 reciprocals (mixed form multiplies where the reference divides)
  const int *eoeP;                // the TRiSK rows (eoe, w) padded to EOE_MAX entries per edge, pads id 0 weight 0
  const double *wP;
  const float *wP32;
  // neighbour staging of the slow tendency: block c of THREADS edges names the distinct edges sList[sOff[c] ..
  // sOff[c + 1]) in its rows; sLoc (E x EOE_MAX) gives each row entry's position in that list; sMax the longest list
  const int *sOff, *sList;
  const int16_t *sLoc;
  int sMax;
};

// A cell's six slots of a per-cell table (int32: 24-byte rows; int8: 6-byte rows). Each table is its own allocation,
// so rows are 8-byte (int32) or 2-byte (int8) aligned: three vector loads instead of six scalar ones, which in a
// thread-per-cell pass cuts the L1 sector lookups of the row from six per thread to three.
__device__ __forceinline__ void slots6(const int *__restrict__ t, int i, int out[6]) {
  const int2 *p = reinterpret_cast<const int2 *>(t + (size_t)i * 6);
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int2 v = p[q];
    out[2 * q] = v.x;
    out[2 * q + 1] = v.y;
  }
}

__device__ __forceinline__ void signs6(const int8_t *__restrict__ t, int i, int out[6]) {
  const char2 *p = reinterpret_cast<const char2 *>(t + (size_t)i * 6);
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const char2 v = p[q];
    out[2 * q] = (signed char)v.x;
    out[2 * q + 1] = (signed char)v.y;
  }
}

// Edge e's padded TRiSK row: ids as five 8-byte loads, weights as five 16-byte (FP64) or 8-byte (FP32) loads.
__device__ __forceinline__ void trisk_row(const GridDev &g, int e, int ix[EOE_MAX], double wv[EOE_MAX]) {
  static_assert(EOE_MAX % 2 == 0, "padded TRiSK rows are read in pairs");
  const int2 *pi = reinterpret_cast<const int2 *>(g.eoeP + (size_t)e * EOE_MAX);
  const double2 *pw = reinterpret_cast<const double2 *>(g.wP + (size_t)e * EOE_MAX);
#pragma unroll
  for (int q = 0; q < EOE_MAX / 2; q++) {
    const int2 a = pi[q];
    const double2 b = pw[q];
    ix[2 * q] = a.x; ix[2 * q + 1] = a.y;
    wv[2 * q] = b.x; wv[2 * q + 1] = b.y;
  }
}

__device__ __forceinline__ void trisk_row(const GridDev &g, int e, int ix[EOE_MAX], float wv[EOE_MAX]) {
  const int2 *pi = reinterpret_cast<const int2 *>(g.eoeP + (size_t)e * EOE_MAX);
  const float2 *pw = reinterpret_cast<const float2 *>(g.wP32 + (size_t)e * EOE_MAX);
#pragma unroll
  for (int q = 0; q < EOE_MAX / 2; q++) {
    const int2 a = pi[q];
    const float2 b = pw[q];
    ix[2 * q] = a.x; ix[2 * q + 1] = a.y;
    wv[2 * q] = b.x; wv[2 * q + 1] = b.y;
  }
}

// Edge e's row entries as positions in its block's staged neighbour list (five 4-byte loads).
__device__ __forceinline__ void trisk_loc(const GridDev &g, int e, int loc[EOE_MAX]) {
  const short2 *p = reinterpret_cast<const short2 *>(g.sLoc + (size_t)e * EOE_MAX);
#pragma unroll
  for (int q = 0; q < EOE_MAX / 2; q++) {
    const short2 v = p[q];
    loc[2 * q] = v.x;
    loc[2 * q + 1] = v.y;
  }
}

__device__ __forceinline__ void trisk_weights(const GridDev &g, int e, double wv[EOE_MAX]) {
  const double2 *pw = reinterpret_cast<const double2 *>(g.wP + (size_t)e * EOE_MAX);
#pragma unroll
  for (int q = 0; q < EOE_MAX / 2; q++) {
    const double2 b = pw[q];
    wv[2 * q] = b.x; wv[2 * q + 1] = b.y;
  }
}

__device__ __forceinline__ void trisk_weights(const GridDev &g, int e, float wv[EOE_MAX]) {
  const float2 *pw = reinterpret_cast<const float2 *>(g.wP32 + (size_t)e * EOE_MAX);
#pragma unroll
  for (int q = 0; q < EOE_MAX / 2; q++) {
    const float2 b = pw[q];
    wv[2 * q] = b.x; wv[2 * q + 1] = b.y;
  }
}

// Scratch and parameters of one Layers object (reference layers.py:36-92), by value in kernel parameters.
struct LayersDev {
  GridDev g;
  int L, precision;
  double grav, nu4, floor_, div_damp, thin, vmix, vmix_cd;
  double gp[LMAX], drag[LMAX], stress[LMAX];
  const double *b, *fV;
  double *Gc;                                // the fast mode's coefficient per cell: g, or for air layers R T_s / mu
  double *B, *q, *Tp, *F, *scale, *G, *He, *ubs, *ub0, *ub, *acc, *eta0, *eta, *eta_prev;
  double *h1, *h2, *u1, *u2, *D1, *Z1, *L1, *L2, *hedge, *diss, *pk;
  double *ub2;                               // second exchange buffer of the tiled fast loop
  double *cw;                                // grid-wide fast loop: per cell and slot sign l_e H_e (N x 6)
  double *red;                               // reduction scratch (substeps)
  // air layers (h = mass per area, theta per layer): their constants and scratch
  int air;
  double cpa, kap, rda, p0, thin_wind;
  double *hold;                              // the exchange hook's h before it (L x N)
  // option branches (reference layers.py:36-90; null / 0 when off): thin walls (E mask, 0 = closed), the squeezed-layer
  // shelf and its bed flags ob (L x N), per-cell buoyancy sig with the layers' mid-heights zm (L x N), the tide potential
  // (N), the bottom layer's quadratic drag cd_bot and the internal tide's drag cbot (E)
  double shelf, cd_bot;
  const double *wall, *sig, *tide, *cbot;
  double *zm, *ob;
  double *S, *pibar, *muf, *phi, *uf, *accL;
  // mixed-form scratch (allocated for ISW_MIXED only): FP32 stage winds and operators; the fast loop in deviation form
  // (deta = eta - eta0, dub = ubar - ubar0) with its exchange buffers; pk4 = per edge and layer (h_e, u, q_e, 0)
  float *u32, *u1f, *u2f, *D1f, *Z1f, *L1f, *L2f, *q32, *Tp32, *G32, *He32, *ubs32, *Gc32;
  float *dub, *deta, *deprev, *xeta[2], *xdub[2];
  float *cw32;                               // grid-wide fast loop, per cell (N x 8): sign l_e H_e / A per slot, c0 / A, Gc
  float2 *Gr32;                              // per edge (G, 1/d_e): the grid-wide edge sub-step's two operands in one load
  float *F32, *scale32;                      // mixed form: stored layer fluxes (L x E) and limiter factors (L x N)
  double *wsum;                              // mixed form, grid-wide fast loop: W, the weighted sum of Y (N)
  float4 *pk4;
};

// Arguments of one RK3 stage (reference layers.py:129-183).
struct StageArgs {
  const double *hs, *us, *h0, *u0;
  double *hn, *un, *Fm;
  double cdt, dt, tau, inv_n;
  int n;                                     // fast sub-steps of this stage
};

inline int blocks_for(long long n, int threads = THREADS) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace isw

struct isw_grid {
  int device;
  int n;
  isw::GridDev d;
  std::vector<void *> allocs;
  double dmin;                   // smallest edge spacing (Layers.dmin)
  std::vector<int32_t> h_nbr, h_cellEdge, h_eI, h_eJ;   // host copies the fast-loop tiles are built from
  std::vector<int8_t> h_cellSign;
  std::vector<double> h_de, h_le, h_areaCell;
};
