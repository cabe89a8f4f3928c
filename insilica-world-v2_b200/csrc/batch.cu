// Batched step: every registered stack (a Layers object with its state, optionally its Transport and tracers)
// advanced by one time-split RK3 step, its receiving masses and one FCT transport step, as ONE CUDA graph per step.
//
// Each phase is one kernel over every stack at once: a table of chunks (stack, up to 256 items of its cells, edges,
// vertices or tracer rows), one chunk per block, the stack's descriptor staged in shared memory. Stacks may sit on
// different grids and have different layer counts. The barotropic fast loop of a stage is one cooperative kernel over
// shared-memory tiles (tiles.cuh): k sub-steps per grid-wide exchange instead of two launches per sub-step; stacks
// whose tiles would not fit in shared memory take the sub-steps as grid-wide kernels instead. The phase functions are
// the per-call path's (layers_fp64.cuh, transport_fp64.cuh), so every stack's result is bit-identical to stepping it
// alone, whatever else shares the launches.
//
// Per step: init (+ first Laplacian pass) | lap e | lap cv | lap e | per stage: A, E, S, fast loop, C, D |
// vmix + transport P1 (with the receiving masses) | P2 | P3 | P4 (and M <- M1).
//
// The tile kernel's grid barrier waits with an iteration-bounded, time-bounded spin (globaltimer): if a wait runs out
// it records ISW_ETIMEOUT in the batch's status word and every block returns; the host reads the status.
#include <cuda/atomic>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "handles.cuh"
#include "layers_fp64.cuh"
#include "tiles.cuh"
#include "transport_fp64.cuh"

namespace isw {
namespace {


struct TileSetDev {
  int P, k;
  const int *cell_off, *edge_off, *cells, *edges, *ncnt, *ecnt, *eown;
  const int16_t *cedge, *eIl, *eJl;
  const double *ade, *ale, *aarea;            // d_e, l_e per local edge and the area per local cell, in local order
};

struct StackDesc {
  LayersDev M;
  TransportDev T;
  TrArgs tr;                 // M0 = the stack's M, M1, Fm, tracers, L, rows, beta
  double *h, *u, *Fm, *Mm;
  double dt;
  int L, has_tr, tiled;
  int n[3];
  double cdt[3], tau[3], inv_n[3];
  TileSetDev tiles;
};

struct Chunk {
  int s, begin, end;
};

struct TileRef {
  int s, p;
};

struct Sched {
  const Chunk *cell, *edge, *vert, *rows;
  int ncell, nedge, nvert, nrows;
};

struct GridBarrier {
  unsigned count, gen;
};

__device__ __forceinline__ long long globaltimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Block-wide grid barrier with a bounded wait. Returns false once any block has recorded a failure.
__device__ bool grid_sync(GridBarrier *b, int *status, long long timeout_ns, int skip_arrive) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(b->gen), cnt(b->count);
    cuda::atomic_ref<int, cuda::thread_scope_device> st(*status);
    const unsigned g0 = gen.load(cuda::memory_order_acquire);
    __threadfence();
    if (!skip_arrive && cnt.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.fetch_add(1u, cuda::memory_order_release);
    } else {
      const long long t0 = globaltimer();
      unsigned it = 0;
      while (gen.load(cuda::memory_order_acquire) == g0) {
        ++it;
        if ((it & 63) == 0) {
          if (st.load(cuda::memory_order_relaxed) != 0) { ok = 0; break; }
          if (globaltimer() - t0 > timeout_ns) {
            int z = 0;
            st.compare_exchange_strong(z, (int)ISW_ETIMEOUT, cuda::memory_order_relaxed);
            ok = 0;
            break;
          }
        }
        if (it > (1u << 30)) { ok = 0; break; }
      }
    }
    __threadfence();
    if (st.load(cuda::memory_order_relaxed) != 0) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

#define ISW_BATCH_L(LV, LMAXK, CALL)                                                            \
  do {                                                                                          \
    switch (LV) {                                                                               \
      case 1: { constexpr int LL = 1; CALL; } break;                                            \
      case 2: if (LMAXK >= 2) { constexpr int LL = 2 <= LMAXK ? 2 : 1; CALL; } break;           \
      case 3: if (LMAXK >= 3) { constexpr int LL = 3 <= LMAXK ? 3 : 1; CALL; } break;           \
      case 4: if (LMAXK >= 4) { constexpr int LL = 4 <= LMAXK ? 4 : 1; CALL; } break;           \
      case 5: if (LMAXK >= 5) { constexpr int LL = 5 <= LMAXK ? 5 : 1; CALL; } break;           \
      case 6: if (LMAXK >= 6) { constexpr int LL = 6 <= LMAXK ? 6 : 1; CALL; } break;           \
      case 7: if (LMAXK >= 7) { constexpr int LL = 7 <= LMAXK ? 7 : 1; CALL; } break;           \
      case 8: if (LMAXK >= 8) { constexpr int LL = 8 <= LMAXK ? 8 : 1; CALL; } break;           \
      default: break;                                                                           \
    }                                                                                           \
  } while (0)

__device__ __forceinline__ StageArgs stage_args(const StackDesc &d, int st) {
  StageArgs a;
  a.h0 = d.h;
  a.u0 = d.u;
  a.hs = st == 0 ? d.h : st == 1 ? d.M.h1 : d.M.h2;
  a.us = st == 0 ? d.u : st == 1 ? d.M.u1 : d.M.u2;
  a.hn = st == 0 ? d.M.h1 : st == 1 ? d.M.h2 : d.h;
  a.un = st == 0 ? d.M.u1 : st == 1 ? d.M.u2 : d.u;
  a.Fm = st == 2 ? d.Fm : nullptr;
  a.cdt = d.cdt[st];
  a.dt = d.dt;
  a.tau = d.tau[st];
  a.inv_n = d.inv_n[st];
  a.n = d.n[st];
  return a;
}

// The block's stack descriptor, staged in shared memory (one chunk per block, so one stack per block).
__device__ __forceinline__ const StackDesc &stage_desc(const StackDesc *S, int s) {
  __shared__ __align__(16) unsigned char buf[sizeof(StackDesc)];
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(S + s);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(buf);
  for (int w = threadIdx.x; w < (int)(sizeof(StackDesc) / 8); w += blockDim.x) dst[w] = src[w];
  __syncthreads();
  return *reinterpret_cast<const StackDesc *>(buf);
}

enum Phase { PH_INIT, PH_LAPE1, PH_LAPCV, PH_LAPE2, PH_A, PH_E, PH_S, PH_ETA, PH_U, PH_C, PH_D, PH_POST, PH_P2, PH_P3, PH_P4 };

// Domains of a phase, in block order: which chunk tables its blocks walk.
template <int PH>
struct Dom {
  static constexpr bool cell = PH == PH_INIT || PH == PH_LAPCV || PH == PH_A || PH == PH_ETA || PH == PH_C || PH == PH_D;
  static constexpr bool edge = PH == PH_INIT || PH == PH_LAPE1 || PH == PH_LAPE2 || PH == PH_E || PH == PH_S || PH == PH_U ||
                               PH == PH_D || PH == PH_POST;
  static constexpr bool vert = PH == PH_INIT || PH == PH_LAPCV || PH == PH_A;
  static constexpr bool rows = PH == PH_POST || PH == PH_P2 || PH == PH_P3 || PH == PH_P4;
};

template <int PH, int LMAXK>
__global__ void __launch_bounds__(THREADS) k_phase(const StackDesc *__restrict__ S, const Sched sc, int st, int j) {
  int b = blockIdx.x;
  int kind = -1;
  Chunk ch{0, 0, 0};
  if (Dom<PH>::cell) { if (b < sc.ncell) { kind = 0; ch = sc.cell[b]; } else b -= sc.ncell; }
  if (kind < 0 && Dom<PH>::edge) { if (b < sc.nedge) { kind = 1; ch = sc.edge[b]; } else b -= sc.nedge; }
  if (kind < 0 && Dom<PH>::vert) { if (b < sc.nvert) { kind = 2; ch = sc.vert[b]; } else b -= sc.nvert; }
  if (kind < 0 && Dom<PH>::rows) { if (b < sc.nrows) { kind = 3; ch = sc.rows[b]; } else b -= sc.nrows; }
  if (kind < 0) return;
  const StackDesc &d = stage_desc(S, ch.s);
  const int i = ch.begin + (int)threadIdx.x;
  if (i >= ch.end) return;
  const LayersDev &M = d.M;
  if (PH == PH_INIT) {
    if (kind == 0) {
      ISW_BATCH_L(d.L, LMAXK, fp64::eta0_cell<LL>(M, d.h, i));
      if (M.nu4 != 0) ISW_BATCH_L(d.L, LMAXK, fp64::div_cell<LL>(M, d.u, i));
    } else if (kind == 1) {
      ISW_BATCH_L(d.L, LMAXK, fp64::ubar0_edge<LL>(M, d.h, d.u, i));
    } else if (M.nu4 != 0) {
      ISW_BATCH_L(d.L, LMAXK, fp64::curl_vertex<LL>(M, d.u, i));
    }
  } else if (PH == PH_LAPE1 || PH == PH_LAPE2) {
    if (M.nu4 != 0) ISW_BATCH_L(d.L, LMAXK, fp64::lap_edge<LL>(M, PH == PH_LAPE1 ? M.L1 : M.L2, i));
  } else if (PH == PH_LAPCV) {
    if (M.nu4 != 0) {
      if (kind == 0) ISW_BATCH_L(d.L, LMAXK, fp64::div_cell<LL>(M, M.L1, i));
      else ISW_BATCH_L(d.L, LMAXK, fp64::curl_vertex<LL>(M, M.L1, i));
    }
  } else if (PH == PH_A) {
    const StageArgs a = stage_args(d, st);
    if (kind == 0) ISW_BATCH_L(d.L, LMAXK, fp64::bern_cell<LL>(M, a.hs, a.us, i));
    else ISW_BATCH_L(d.L, LMAXK, fp64::pv_vertex<LL>(M, a.hs, a.us, i));
  } else if (PH == PH_E) {
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::edge_hq<LL>(M, a.hs, a.us, i));
  } else if (PH == PH_S) {
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::slow_edge<LL>(M, a.us, a.cdt, i));
  } else if (PH == PH_ETA) {
    if (!d.tiled && j < d.n[st]) fp64::bt_eta_cell(M, d.tau[st], i);
  } else if (PH == PH_U) {
    if (!d.tiled && j < d.n[st]) fp64::bt_u_edge(M, d.tau[st], i);
  } else if (PH == PH_C) {
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::scale_cell<LL>(M, a, i));
  } else if (PH == PH_D) {
    const StageArgs a = stage_args(d, st);
    if (kind == 0) ISW_BATCH_L(d.L, LMAXK, fp64::h_cell<LL>(M, a, i));
    else ISW_BATCH_L(d.L, LMAXK, fp64::u_edge<LL>(M, a, i));
  } else if (PH == PH_POST) {
    if (kind == 1) {
      if ((M.vmix != 0 || M.vmix_cd != 0) && d.L > 1) ISW_BATCH_L(d.L, LMAXK, fp64::vmix_edge<LL>(M, d.h, d.u, d.dt, i));
    } else {
      ISW_BATCH_L(d.L, LMAXK, fp64::tr_p1<LL>(d.T, d.tr, 3, true, i / M.g.N, i % M.g.N));
    }
  } else if (PH == PH_P2) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_p2<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P3) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_p3<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P4) {
    const int j = i / M.g.N, c = i % M.g.N;
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_p4<LL>(d.T, d.tr, j, c));
    if (j == 0)
      for (int l = 0; l < d.L; l++) d.Mm[(size_t)l * M.g.N + c] = d.tr.M1[(size_t)l * M.g.N + c];
  }
}

// The barotropic fast loop of stage `st` for every tiled stack (reference layers.cu:366-388, layers.py:168-175), one
// block per tile, all tiles co-resident (cooperative launch). Same arithmetic as fp64::bt_eta_cell / bt_u_edge.
// Exchange buffers (the owned values each round publishes, double-buffered by round parity): eta / eta_prev for the
// surface and ub2 / F for the barotropic wind (F, the layer fluxes, is not in use during the fast loop). The final
// barotropic wind and its accumulated sum go to ub and acc, which no round reads.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fast(const StackDesc *__restrict__ S, const TileRef *__restrict__ refs, int st,
                                                    int rounds, GridBarrier *bar, int *status, long long timeout_ns,
                                                    int fault_block) {
  extern __shared__ __align__(16) unsigned char smem[];
  const TileRef tr = refs[blockIdx.x];
  const StackDesc &d = S[tr.s];
  const LayersDev &M = d.M;
  const GridDev &g = M.g;
  const TileSetDev &T = d.tiles;
  const int p = tr.p, k = T.k;
  const int c0 = T.cell_off[p], nc = T.cell_off[p + 1] - c0;
  const int e0 = T.edge_off[p], ne = T.edge_off[p + 1] - e0;
  const int eown = T.eown[p];
  const int *cells = T.cells + c0;
  const int *edges = T.edges + e0;
  const int *ncnt = T.ncnt + (size_t)p * (k + 1);
  const int *ecnt = T.ecnt + (size_t)p * (k + 1);
  // shared memory: doubles first, then 16-bit ids
  double *eta = reinterpret_cast<double *>(smem);
  double *eprev = eta + nc;
  double *area = eprev + nc;
  double *gc = area + nc;
  double *ub = gc + nc;
  double *G = ub + ne;
  double *de = G + ne;
  double *lh = de + ne;                    // l_e H_e: with the cell's sign, the reference's (sign * l_e) * H_e
  double *acc = lh + ne;                   // owned edges only
  int16_t *cedge = reinterpret_cast<int16_t *>(acc + eown);
  int16_t *eIl = cedge + (size_t)nc * 6;
  int16_t *eJl = eIl + ne;
  const int skip = (int)blockIdx.x == fault_block;
  const int n = d.n[st];
  const double tau = d.tau[st], gam = M.div_damp;
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    const int gi = cells[c];
    eta[c] = M.eta0[gi];
    area[c] = T.aarea[c0 + c];
    gc[c] = M.Gc[gi];
  }
  for (int w = threadIdx.x; w < nc * 6; w += blockDim.x) cedge[w] = T.cedge[(size_t)c0 * 6 + w];
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const int ge = edges[e];
    ub[e] = M.ub0[ge];
    G[e] = M.G[ge];
    de[e] = T.ade[e0 + e];
    lh[e] = T.ale[e0 + e] * M.He[ge];
    if (e < eown) acc[e] = 0.0;
    eIl[e] = T.eIl[e0 + e];
    eJl[e] = T.eJl[e0 + e];
  }
  const int nown = ncnt[0];
  for (int r = 0; r < rounds; r++) {
    const int K = min(k, n - r * k);        // sub-steps of this stack in this round (<= 0: idle, barriers only)
    if (r > 0) {
      if (!grid_sync(bar, status, timeout_ns, skip)) return;
      if (K > 0) {                         // round r reads what round r - 1 published: buffer (r - 1) & 1
        const double *xe = ((r - 1) & 1) ? M.eta_prev : M.eta;
        const double *xu = ((r - 1) & 1) ? M.F : M.ub2;
        // only the halo: the owned cells and edges already hold exactly what was published
        for (int c = nown + threadIdx.x; c < nc; c += blockDim.x) eta[c] = xe[cells[c]];
        for (int e = eown + threadIdx.x; e < ne; e += blockDim.x) ub[e] = xu[edges[e]];
      }
    }
    __syncthreads();
    for (int m = 1; m <= K; m++) {
      const int cn = ncnt[K - m + 1];
      for (int c = threadIdx.x; c < cn; c += blockDim.x) {
        const double e0v = eta[c];
        eprev[c] = e0v;
        double div = 0;
        int vs[6];
#pragma unroll
        for (int s = 0; s < 6; s++) vs[s] = cedge[c * 6 + s];
#pragma unroll
        for (int s = 0; s < 6; s++) {
          const int v = vs[s];
          if (v == 0) continue;
          const int le_ = (v > 0 ? v : -v) - 1;
          const double cf = v > 0 ? lh[le_] : -lh[le_];
          div += cf * ub[le_];
        }
        eta[c] = e0v - (tau * div) / area[c];
      }
      __syncthreads();
      const int en = ecnt[K - m];
      for (int e = threadIdx.x; e < en; e += blockDim.x) {
        const double v = ub[e];
        if (e < eown) acc[e] += v;
        const int i = eIl[e], jj = eJl[e];
        const double ej = gc[jj] * (eta[jj] + gam * (eta[jj] - eprev[jj]));
        const double ei = gc[i] * (eta[i] + gam * (eta[i] - eprev[i]));
        ub[e] = v + tau * ((-(ej - ei)) / de[e] + G[e]);
      }
      __syncthreads();
    }
    if (r + 1 < rounds && K > 0) {           // publish the owned values for the neighbours' next round: buffer r & 1
      double *xe = (r & 1) ? M.eta_prev : M.eta;
      double *xu = (r & 1) ? M.F : M.ub2;
      for (int c = threadIdx.x; c < nown; c += blockDim.x) xe[cells[c]] = eta[c];
      for (int e = threadIdx.x; e < eown; e += blockDim.x) xu[edges[e]] = ub[e];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < eown; e += blockDim.x) {
    M.ub[edges[e]] = ub[e];
    M.acc[edges[e]] = acc[e];
  }
}

}  // namespace
}  // namespace isw

using namespace isw;

struct BatchSlot {
  bool used = false;
  isw_layers *layers = nullptr;
  isw_transport *tr = nullptr;
  double *h = nullptr, *u = nullptr, *Fm = nullptr, *M = nullptr, *M1 = nullptr;
  double *tracers[TRMAX] = {};
  int ntr = 0;
  double dt = 0;
  int nfast = 0;
};

struct TileCache {
  TileSetDev dev{};
  TileSetHost host;
  std::vector<void *> allocs;
};

struct isw_batch {
  int device;
  std::vector<BatchSlot> slots;
  bool dirty = true;
  StackDesc *d_desc = nullptr;
  Chunk *d_chunks = nullptr;
  TileRef *d_refs = nullptr;
  Sched sc{};
  int lmax = 1, nstacks = 0, ntiles = 0, rounds[3] = {0, 0, 0}, nsub[3] = {0, 0, 0}, kused = 0;
  int any_nu4 = 0, any_vmix = 0, any_tr = 0, any_untiled = 0;
  size_t fast_smem = 0;
  int fast_bps = 2;                           // tile blocks per SM: 2 (512 threads each) or 1 (1024 threads)
  GridBarrier *bar = nullptr;
  int *status = nullptr;
  int tile_k = 8;
  int tiles_enabled = 1;
  std::map<std::tuple<const isw_grid *, int, int>, std::unique_ptr<TileCache>> tiles;
  std::map<std::pair<const isw_grid *, int>, std::vector<int32_t>> parts;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  int sms = 0;
};

namespace {

template <class F>
int guarded(F f) {
  try {
    f();
    return ISW_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return ISW_ENOMEM;
  }
}

constexpr long long DEFAULT_TIMEOUT_NS = 2000000000LL;   // 2 s: far beyond any stage; only a broken grid reaches it
constexpr size_t SMEM_TWO = 112 * 1024;                  // per tile block when two share an SM
constexpr size_t SMEM_ONE = 224 * 1024;                  // per tile block alone on an SM
constexpr int K_PROBE = 8;                               // the largest exchange interval considered

template <class T>
T *dupload(std::vector<void *> &allocs, const std::vector<T> &v) {
  void *p = nullptr;
  ISW_CUDA(cudaMalloc(&p, sizeof(T) * (v.empty() ? 1 : v.size())));
  allocs.push_back(p);
  if (!v.empty()) ISW_CUDA(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return (T *)p;
}

const std::vector<int32_t> &partition_for(isw_batch *b, const isw_grid *g, int P);

const std::vector<int32_t> &partition_for(isw_batch *b, const isw_grid *g, int P) {
  auto key = std::make_pair(g, P);
  auto it = b->parts.find(key);
  if (it != b->parts.end()) return it->second;
  return b->parts[key] = partition_cells(g->d.N, g->h_nbr.data(), P);
}

TileCache *tiles_for(isw_batch *b, const isw_grid *g, int P, int k) {
  auto key = std::make_tuple(g, P, k);
  auto it = b->tiles.find(key);
  if (it != b->tiles.end()) return it->second.get();
  auto c = std::make_unique<TileCache>();
  c->host = build_tiles(g->d.N, g->d.E, g->h_nbr.data(), g->h_cellEdge.data(), g->h_cellSign.data(), g->h_eI.data(),
                        g->h_eJ.data(), partition_for(b, g, P), P, k);
  const TileSetHost &h = c->host;
  TileSetDev &t = c->dev;
  t.P = P;
  t.k = k;
  t.cell_off = dupload(c->allocs, h.cell_off);
  t.edge_off = dupload(c->allocs, h.edge_off);
  t.cells = dupload(c->allocs, h.cells);
  t.edges = dupload(c->allocs, h.edges);
  t.ncnt = dupload(c->allocs, h.ncnt);
  t.ecnt = dupload(c->allocs, h.ecnt);
  t.eown = dupload(c->allocs, h.eown);
  t.cedge = dupload(c->allocs, h.cedge);
  t.eIl = dupload(c->allocs, h.eIl);
  t.eJl = dupload(c->allocs, h.eJl);
  std::vector<double> ade(h.edges.size()), ale(h.edges.size()), aarea(h.cells.size());
  for (size_t q = 0; q < h.edges.size(); q++) { ade[q] = g->h_de[h.edges[q]]; ale[q] = g->h_le[h.edges[q]]; }
  for (size_t q = 0; q < h.cells.size(); q++) aarea[q] = g->h_areaCell[h.cells[q]];
  t.ade = dupload(c->allocs, ade);
  t.ale = dupload(c->allocs, ale);
  t.aarea = dupload(c->allocs, aarea);
  TileCache *out = c.get();
  b->tiles[key] = std::move(c);
  return out;
}

// The largest k' <= the probe's k whose largest tile fits `budget` bytes of shared memory (0 if none).
int fitting_k(const TileSetHost &h, size_t budget) {
  for (int kk = h.k; kk >= 1; kk--) {
    size_t worst = 0;
    for (int p = 0; p < h.P; p++) {
      const size_t nc = h.ncnt[(size_t)p * (h.k + 1) + kk], ne = h.ecnt[(size_t)p * (h.k + 1) + kk];
      worst = std::max(worst, tile_smem_bytes(nc, ne, h.eown[p]));
    }
    if (worst <= budget) return kk;
  }
  return 0;
}

int kernel_lmax(int L) { return L <= 2 ? 2 : L <= 3 ? 3 : L <= 5 ? 5 : 8; }

void rebuild(isw_batch *b) {
  std::vector<StackDesc> desc;
  std::vector<Chunk> cell, edge, vert, rows;
  std::vector<TileRef> refs;
  int nsub[3] = {0, 0, 0};
  int any_nu4 = 0, any_vmix = 0, any_tr = 0, any_untiled = 0, lmax = 1;
  size_t fast_smem = 0;
  const double cs[3] = {1.0 / 3.0, 1.0 / 2.0, 1.0};
  // the tiling: per stack P tiles (its share of the tile slots by cell count) and one exchange interval k for all
  // stacks, the largest that fits the shared memory of one or of two tile blocks per SM
  long long cells_total = 0;
  int used = 0;
  for (auto &sl : b->slots)
    if (sl.used) { cells_total += sl.layers->grid->d.N; used++; }
  std::vector<int> Pbest(b->slots.size(), 0);
  int kbest = 0, bps_best = 2;
  if (b->tiles_enabled && used > 0) {
    for (int bps = 2; bps >= 1; bps--) {
      const size_t budget = bps == 2 ? SMEM_TWO : SMEM_ONE;
      const int slots = b->sms * bps;
      std::vector<int> P(b->slots.size(), 0);
      int kmin = b->tile_k;
      bool any = false;
      for (size_t q = 0; q < b->slots.size(); q++) {
        const BatchSlot &sl = b->slots[q];
        if (!sl.used) continue;
        const int N = sl.layers->grid->d.N;
        const int Pq = std::max(1, (int)((long long)slots * N / std::max(1LL, cells_total)));
        if (Pq * 16 > N) continue;             // tiles of at least 16 owned cells
        const int kf = fitting_k(tiles_for(b, sl.layers->grid, Pq, std::min(K_PROBE, b->tile_k))->host, budget);
        if (kf == 0) continue;
        P[q] = Pq;
        kmin = std::min(kmin, kf);
        any = true;
      }
      if (any && kmin > kbest) {
        kbest = kmin;
        bps_best = bps;
        Pbest = P;
      }
    }
  }
  for (auto &sl : b->slots) {
    if (!sl.used) continue;
    StackDesc d;
    std::memset(&d, 0, sizeof(d));
    d.M = sl.layers->d;
    d.h = sl.h; d.u = sl.u; d.Fm = sl.Fm; d.Mm = sl.M;
    d.dt = sl.dt;
    d.L = d.M.L;
    lmax = std::max(lmax, d.L);
    for (int st = 0; st < 3; st++) {
      const double c = cs[st];
      const double cn = std::ceil(c * sl.nfast);
      d.n[st] = cn > 1 ? (int)cn : 1;
      d.cdt[st] = c * sl.dt;
      d.tau[st] = c * sl.dt / d.n[st];
      d.inv_n[st] = 1.0 / d.n[st];
      nsub[st] = std::max(nsub[st], d.n[st]);
    }
    if (d.M.nu4 != 0) any_nu4 = 1;
    if ((d.M.vmix != 0 || d.M.vmix_cd != 0) && d.L > 1) any_vmix = 1;
    if (sl.tr) {
      d.has_tr = 1;
      any_tr = 1;
      d.T = sl.tr->d;
      d.tr.M0 = sl.M; d.tr.M1 = sl.M1; d.tr.Fm = sl.Fm; d.tr.L = d.L; d.tr.rows = sl.ntr * d.L; d.tr.beta = sl.tr->beta;
      for (int j = 0; j < sl.ntr; j++) d.tr.tr[j] = sl.tracers[j];
    }
    const int s = (int)desc.size();
    d.tiled = 0;
    const size_t q = (size_t)(&sl - &b->slots[0]);
    if (kbest > 0 && Pbest[q] > 0) {
      TileCache *tc = tiles_for(b, sl.layers->grid, Pbest[q], kbest);
      d.tiled = 1;
      d.tiles = tc->dev;
      fast_smem = std::max(fast_smem, tc->host.smem);
      for (int p = 0; p < Pbest[q]; p++) refs.push_back(TileRef{s, p});
    }
    if (!d.tiled) any_untiled = 1;
    auto chunks = [&](std::vector<Chunk> &v, int n) {
      for (int i = 0; i < n; i += THREADS) v.push_back(Chunk{s, i, std::min(n, i + THREADS)});
    };
    chunks(cell, d.M.g.N);
    chunks(edge, d.M.g.E);
    chunks(vert, d.M.g.NV);
    if (d.has_tr) chunks(rows, sl.ntr * d.M.g.N);       // (tracer, cell) pairs
    desc.push_back(d);
  }
  b->nstacks = (int)desc.size();
  cudaFree(b->d_desc);
  cudaFree(b->d_chunks);
  cudaFree(b->d_refs);
  b->d_desc = nullptr;
  b->d_chunks = nullptr;
  b->d_refs = nullptr;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  b->dirty = false;
  if (desc.empty()) return;
  std::vector<Chunk> all;
  all.insert(all.end(), cell.begin(), cell.end());
  all.insert(all.end(), edge.begin(), edge.end());
  all.insert(all.end(), vert.begin(), vert.end());
  all.insert(all.end(), rows.begin(), rows.end());
  ISW_CUDA(cudaMalloc(&b->d_desc, sizeof(StackDesc) * desc.size()));
  ISW_CUDA(cudaMemcpy(b->d_desc, desc.data(), sizeof(StackDesc) * desc.size(), cudaMemcpyHostToDevice));
  ISW_CUDA(cudaMalloc(&b->d_chunks, sizeof(Chunk) * all.size()));
  ISW_CUDA(cudaMemcpy(b->d_chunks, all.data(), sizeof(Chunk) * all.size(), cudaMemcpyHostToDevice));
  if (!refs.empty()) {
    ISW_CUDA(cudaMalloc(&b->d_refs, sizeof(TileRef) * refs.size()));
    ISW_CUDA(cudaMemcpy(b->d_refs, refs.data(), sizeof(TileRef) * refs.size(), cudaMemcpyHostToDevice));
  }
  Sched &sc = b->sc;
  sc.cell = b->d_chunks;
  sc.ncell = (int)cell.size();
  sc.edge = sc.cell + sc.ncell;
  sc.nedge = (int)edge.size();
  sc.vert = sc.edge + sc.nedge;
  sc.nvert = (int)vert.size();
  sc.rows = sc.vert + sc.nvert;
  sc.nrows = (int)rows.size();
  b->ntiles = (int)refs.size();
  b->fast_smem = fast_smem;
  b->fast_bps = bps_best;
  if (b->ntiles > 0) {                      // every tile block must be resident at once (cooperative launch)
    const void *fn = bps_best == 2 ? (const void *)k_fast<512, 2> : (const void *)k_fast<1024, 1>;
    if (fast_smem > 48 * 1024) ISW_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fast_smem));
    int per = 0;
    ISW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, bps_best == 2 ? 512 : 1024, fast_smem));
    if ((long long)per * b->sms < b->ntiles) {
      b->ntiles = 0;
      any_untiled = 1;
      for (auto &d : desc) d.tiled = 0;
      ISW_CUDA(cudaMemcpy(b->d_desc, desc.data(), sizeof(StackDesc) * desc.size(), cudaMemcpyHostToDevice));
    }
  }
  for (int st = 0; st < 3; st++) {
    b->nsub[st] = nsub[st];
    b->rounds[st] = kbest > 0 ? (nsub[st] + kbest - 1) / kbest : 0;
  b->kused = kbest;
  }
  b->any_nu4 = any_nu4;
  b->any_vmix = any_vmix;
  b->any_tr = any_tr;
  b->any_untiled = any_untiled;
  b->lmax = kernel_lmax(lmax);
}

template <int PH>
void launch_phase(isw_batch *b, cudaStream_t st, int stage, int j) {
  const Sched &sc = b->sc;
  const int nb = (Dom<PH>::cell ? sc.ncell : 0) + (Dom<PH>::edge ? sc.nedge : 0) + (Dom<PH>::vert ? sc.nvert : 0) +
                 (Dom<PH>::rows ? sc.nrows : 0);
  if (nb == 0) return;
  switch (b->lmax) {
    case 2: k_phase<PH, 2><<<nb, THREADS, 0, st>>>(b->d_desc, sc, stage, j); break;
    case 3: k_phase<PH, 3><<<nb, THREADS, 0, st>>>(b->d_desc, sc, stage, j); break;
    case 5: k_phase<PH, 5><<<nb, THREADS, 0, st>>>(b->d_desc, sc, stage, j); break;
    default: k_phase<PH, 8><<<nb, THREADS, 0, st>>>(b->d_desc, sc, stage, j); break;
  }
}

void launch_fast(isw_batch *b, cudaStream_t st, int stage, long long timeout_ns, int fault_block) {
  if (b->ntiles == 0) return;
  ISW_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(GridBarrier), st));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)b->ntiles);
  cfg.blockDim = dim3(b->fast_bps == 2 ? 512 : 1024);
  cfg.dynamicSmemBytes = b->fast_smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (b->fast_bps == 2)
    ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast<512, 2>, (const StackDesc *)b->d_desc, (const TileRef *)b->d_refs, stage,
                                b->rounds[stage], b->bar, b->status, timeout_ns, fault_block));
  else
    ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast<1024, 1>, (const StackDesc *)b->d_desc, (const TileRef *)b->d_refs, stage,
                                b->rounds[stage], b->bar, b->status, timeout_ns, fault_block));
}

// The launches of one step, in order.
void enqueue(isw_batch *b, cudaStream_t st) {
  launch_phase<PH_INIT>(b, st, 0, 0);
  if (b->any_nu4) {
    launch_phase<PH_LAPE1>(b, st, 0, 0);
    launch_phase<PH_LAPCV>(b, st, 0, 0);
    launch_phase<PH_LAPE2>(b, st, 0, 0);
  }
  for (int s = 0; s < 3; s++) {
    launch_phase<PH_A>(b, st, s, 0);
    launch_phase<PH_E>(b, st, s, 0);
    launch_phase<PH_S>(b, st, s, 0);
    launch_fast(b, st, s, DEFAULT_TIMEOUT_NS, -1);
    if (b->any_untiled)
      for (int j = 0; j < b->nsub[s]; j++) {
        launch_phase<PH_ETA>(b, st, s, j);
        launch_phase<PH_U>(b, st, s, j);
      }
    launch_phase<PH_C>(b, st, s, 0);
    launch_phase<PH_D>(b, st, s, 0);
  }
  if (b->any_vmix || b->any_tr) launch_phase<PH_POST>(b, st, 0, 0);
  if (b->any_tr) {
    launch_phase<PH_P2>(b, st, 0, 0);
    launch_phase<PH_P3>(b, st, 0, 0);
    launch_phase<PH_P4>(b, st, 0, 0);
  }
  ISW_CUDA(cudaGetLastError());
}

void prepare(isw_batch *b) {
  if (b->dirty) rebuild(b);
}

void step(isw_batch *b, cudaStream_t st) {
  prepare(b);
  if (b->nstacks == 0) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ISW_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {    // inside the caller's capture: queue the launches themselves
    enqueue(b, st);
    return;
  }
  if (!b->exec) {
    cudaGraph_t graph = nullptr;
    ISW_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue(b, b->cap);
    } catch (...) {
      cudaStreamEndCapture(b->cap, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    ISW_CUDA(cudaStreamEndCapture(b->cap, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    ISW_CUDA(ie);
  }
  ISW_CUDA(cudaGraphLaunch(b->exec, st));
}

}  // namespace

extern "C" {

int isw_batch_create(int device, isw_batch **out) {
  return guarded([&] {
    if (!out) fail(ISW_EINVAL, "batch: null output handle");
    ISW_CUDA(cudaSetDevice(device));
    isw_batch *b = new isw_batch();
    b->device = device;
    try {
      ISW_CUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device));
      ISW_CUDA(cudaMalloc(&b->bar, sizeof(GridBarrier)));
      ISW_CUDA(cudaMemset(b->bar, 0, sizeof(GridBarrier)));
      ISW_CUDA(cudaMalloc(&b->status, sizeof(int)));
      ISW_CUDA(cudaMemset(b->status, 0, sizeof(int)));
      ISW_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    } catch (...) {
      cudaFree(b->bar);
      cudaFree(b->status);
      delete b;
      throw;
    }
    *out = b;
  });
}

int isw_batch_destroy(isw_batch *b) {
  if (!b) return ISW_OK;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->cap) cudaStreamDestroy(b->cap);
  cudaFree(b->d_desc);
  cudaFree(b->d_chunks);
  cudaFree(b->d_refs);
  cudaFree(b->bar);
  cudaFree(b->status);
  for (auto &kv : b->tiles)
    for (void *p : kv.second->allocs) cudaFree(p);
  delete b;
  return ISW_OK;
}

int isw_batch_add(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *M, double *M1,
                  double *const *tracers, int ntr, double dt, int nfast, int *slot) {
  return guarded([&] {
    if (!b || !layers || !h || !u || !Fm || !slot) fail(ISW_EINVAL, "batch.add: null argument");
    if (layers->grid->device != b->device) fail(ISW_EINVAL, "batch.add: the stack is on another device");
    if (!(dt > 0) || !std::isfinite(dt) || nfast < 1) fail(ISW_EINVAL, "batch.add: dt must be positive and nfast >= 1");
    if (tr) {
      if (!M || !M1 || !tracers) fail(ISW_EINVAL, "batch.add: transport needs M, M1 and the tracers");
      if (ntr < 1 || ntr > tr->T) fail(ISW_EINVAL, "batch.add: ntr outside 1..tracers of the transport");
      if (tr->L != layers->d.L || tr->grid != layers->grid) fail(ISW_EINVAL, "batch.add: transport and layers differ in grid or L");
    }
    BatchSlot sl;
    sl.used = true;
    sl.layers = layers;
    sl.tr = tr;
    sl.h = h; sl.u = u; sl.Fm = Fm; sl.M = M; sl.M1 = M1;
    sl.ntr = tr ? ntr : 0;
    for (int j = 0; j < sl.ntr; j++) {
      if (!tracers[j]) fail(ISW_EINVAL, "batch.add: null tracer");
      sl.tracers[j] = tracers[j];
    }
    sl.dt = dt;
    sl.nfast = nfast;
    size_t k = 0;
    while (k < b->slots.size() && b->slots[k].used) k++;
    if (k == b->slots.size()) b->slots.push_back(sl);
    else b->slots[k] = sl;
    b->dirty = true;
    *slot = (int)k;
  });
}

int isw_batch_remove(isw_batch *b, int slot) {
  return guarded([&] {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) fail(ISW_EINVAL, "batch.remove: no such slot");
    b->slots[slot] = BatchSlot();
    b->dirty = true;
  });
}

int isw_batch_config(isw_batch *b, int tiles_enabled, int tile_k) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.config: null handle");
    if (tile_k < 1 || tile_k > 32) fail(ISW_EINVAL, "batch.config: tile_k outside 1..32");
    b->tiles_enabled = tiles_enabled ? 1 : 0;
    b->tile_k = tile_k;
    b->dirty = true;
  });
}

int isw_batch_info(isw_batch *b, int *stacks, int *tiles, int *tile_k, long long *smem_bytes) {
  return guarded([&] {
    if (!b || !stacks || !tiles || !tile_k || !smem_bytes) fail(ISW_EINVAL, "batch.info: null argument");
    ISW_CUDA(cudaSetDevice(b->device));
    prepare(b);
    *stacks = b->nstacks;
    *tiles = b->ntiles;
    *tile_k = b->ntiles > 0 ? b->kused : 0;
    *smem_bytes = (long long)b->fast_smem;
  });
}

int isw_batch_step(isw_batch *b, void *stream) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.step: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    step(b, (cudaStream_t)stream);
  });
}

int isw_batch_status(isw_batch *b, void *stream, int reset) {
  int out = ISW_OK;
  const int rc = guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.status: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    int st = 0;
    ISW_CUDA(cudaMemcpyAsync(&st, b->status, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    ISW_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (reset) ISW_CUDA(cudaMemset(b->status, 0, sizeof(int)));
    out = st;
  });
  return rc != ISW_OK ? rc : out;
}

int isw_batch_fault_test(isw_batch *b, long long timeout_ns, void *stream) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.fault_test: null handle");
    if (timeout_ns < 1000000 || timeout_ns > 2000000000LL) fail(ISW_EINVAL, "batch.fault_test: timeout outside 1 ms .. 2 s");
    ISW_CUDA(cudaSetDevice(b->device));
    prepare(b);
    if (b->ntiles == 0) fail(ISW_EUNSUPPORTED, "batch.fault_test: no tiled stack in the batch");
    if (b->rounds[2] < 2) fail(ISW_EUNSUPPORTED, "batch.fault_test: the last stage has no grid barrier");
    launch_fast(b, (cudaStream_t)stream, 2, timeout_ns, 0);
  });
}

}  // extern "C"
