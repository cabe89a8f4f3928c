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
// vmix + FCT stage-1 edge fluxes | P1 (receiving masses, td, p1) | P2E | P2 | P3E | P3 | P4 (and M <- M1).
//
// The tile kernel's grid barrier waits with an iteration-bounded, time-bounded spin (globaltimer): if a wait runs out
// it records ISW_ETIMEOUT in the batch's status word and every block returns. Phase D of the last stage checks every
// new thickness and records ISW_ENOTFINITE for a NaN or Inf. The kernel that records a failure also writes it to a
// mapped host word, and isw_batch_step refuses to run while that word is set (until isw_batch_status resets it), so a
// caller that never polls cannot step on a half-updated state.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "handles.cuh"
#include "layers_air.cuh"
#include "layers_fp64.cuh"
#include "tiles.cuh"
#include "transport_fp64.cuh"

namespace isw {
using namespace bt;
namespace {

// The grid-wide sub-step passes over a wide chunk: PH_ETA's cells, PH_U's / PH_UF's edges (PH_UF also forming the
// layer fluxes on the stack's last sub-step); air stacks and sub-step 0's cell pass (which also forms the slot
// coefficients) item by item.
template <int PH, int LMAXK, bool EXT>
__device__ __forceinline__ void substep_chunk(const StackDesc &d, int st, int j, const Chunk &ch) {
  if (d.tiled || j >= d.n[st]) return;
  const LayersDev &M = d.M;
  const double tau = d.tau[st];
  const int first = ch.begin + (int)threadIdx.x;
  if (EXT && M.air) {
    for (int i = first; i < ch.end; i += THREADS) {
      if (PH == PH_ETA) ISW_BATCH_L(d.L, LMAXK, fp64::af_muphi_cell<LL>(M, tau, i));
      else ISW_BATCH_L(d.L, LMAXK, fp64::af_u_edge<LL>(M, tau, i));
    }
  } else if (PH == PH_ETA) {
    if (j == 0)
      for (int i = first; i < ch.end; i += THREADS) fp64::bt_eta_cell_y(M, tau, 0, i);
    else
      fp64::bt_eta_cells_y<SUB_WC>(M, tau, first, ch.end);
  } else {
    fp64::bt_u_edges_y<SUB_W_FP64, EXT>(M, tau, first, ch.end);
    if (PH == PH_UF && j == d.n[st] - 1) {
      const StageArgs a = stage_args(d, st);
      for (int i = first; i < ch.end; i += THREADS) fp64::flux_edge<EXT>(M, a, M.acc[i], i);
    }
  }
}

// EXT: the kernel also carries the air branch and the option branches (walls, the shelf and its bed flags, per-cell
// buoyancy, the tide, the bottom's drag), instantiated only for batches holding such stacks, so that the plain
// Boussinesq phases keep their register count.
template <int PH, int LMAXK, bool EXT>
__global__ void __launch_bounds__(THREADS) k_phase(const StackDesc *__restrict__ S, const Sched sc, int st, int j) {
  Chunk ch{0, 0, 0};
  const int kind = phase_chunk<PH>(sc, blockIdx.x, ch);
  if (kind < 0) return;
  const StackDesc &d = stage_desc(S, ch.s);
  pdl_wait();
  pdl_trigger();
  if (Dom<PH>::wide) {                       // the grid-wide sub-step passes: a wide chunk, SUB_W items a thread
    substep_chunk<PH, LMAXK, EXT>(d, st, j, ch);
    return;
  }
  const int i = ch.begin + (int)threadIdx.x;
  if (PH == PH_S && d.s_stage) {             // the block stages its rows' distinct neighbour records, then computes
    extern __shared__ __align__(16) double stg[];
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::stage_pk<LL>(d.M, ch.begin / THREADS, stg));
    __syncthreads();
    if (i < ch.end) ISW_BATCH_L(d.L, LMAXK, (fp64::slow_edge<LL, EXT, true>(d.M, a.us, a.cdt, i, nullptr, stg)));
    return;
  }
  if (i >= ch.end) return;
  const LayersDev &M = d.M;
  if (PH == PH_ONBED) {                      // the shelf's bed flags of every layer, before the step's first pass reads them
    if (EXT && M.ob) ISW_BATCH_L(d.L, LMAXK, fp64::onbed_cell<LL>(M, d.h, i));
  } else if (PH == PH_INIT) {
    if (kind == 0) {
      if (EXT && M.air) ISW_BATCH_L(d.L, LMAXK, fp64::air_stiff_cell<LL>(M, d.h, d.theta, i));
      else ISW_BATCH_L(d.L, LMAXK, fp64::eta0_cell<LL>(M, d.h, i));
      if (M.nu4 != 0) ISW_BATCH_L(d.L, LMAXK, fp64::div_cell<LL>(M, d.u, i));
    } else if (kind == 1) {
      if (!(EXT && M.air)) ISW_BATCH_L(d.L, LMAXK, fp64::ubar0_edge<LL, EXT>(M, d.h, d.u, i));
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
    if (kind == 0) {
      if (EXT && M.air) {
        ISW_BATCH_L(d.L, LMAXK, fp64::air_bern_cell<LL>(M, a.hs, a.us, d.theta, i));
        ISW_BATCH_L(d.L, LMAXK, fp64::air_fast_init_cell<LL>(M, a.h0, i));
      } else {
        ISW_BATCH_L(d.L, LMAXK, fp64::bern_cell<LL, EXT>(M, a.hs, a.us, i));
      }
    } else {
      ISW_BATCH_L(d.L, LMAXK, fp64::pv_vertex<LL>(M, a.hs, a.us, i));
    }
  } else if (PH == PH_E) {
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::edge_hq<LL, EXT>(M, a.hs, a.us, i));
    if (EXT && M.air) ISW_BATCH_L(d.L, LMAXK, fp64::air_fast_init_edge<LL>(M, a.u0, i));
  } else if (PH == PH_S) {
    const StageArgs a = stage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, fp64::slow_edge<LL, EXT>(M, a.us, a.cdt, i, EXT && M.air ? d.theta : nullptr));
  } else if (PH == PH_C || PH == PH_CS) {
    const StageArgs a = stage_args(d, st);
    if (EXT && M.air) ISW_BATCH_L(d.L, LMAXK, fp64::air_scale_cell<LL>(M, a, i));
    else if (PH == PH_C) ISW_BATCH_L(d.L, LMAXK, (fp64::scale_cell<LL, EXT>(M, a, i)));
    else ISW_BATCH_L(d.L, LMAXK, fp64::scale_sum_cell<LL>(M, a, i));
  } else if (PH == PH_D) {
    const StageArgs a = stage_args(d, st);
    if (kind == 0) {
      ISW_BATCH_L(d.L, LMAXK, fp64::h_cell<LL>(M, a, i));
      if (st == 2) check_finite_column(d.h, M.g.N, d.L, i, sc.status);
    } else if (EXT && M.air) {
      ISW_BATCH_L(d.L, LMAXK, fp64::air_u_edge<LL>(M, a, i));
    } else {
      ISW_BATCH_L(d.L, LMAXK, fp64::u_edge<LL, EXT>(M, a, i));
    }
  } else if (PH == PH_VMIX) {
    if ((M.vmix != 0 || M.vmix_cd != 0) && d.L > 1) ISW_BATCH_L(d.L, LMAXK, fp64::vmix_edge<LL, EXT>(M, d.h, d.u, d.dt, i));
  } else if (PH == PH_VHEAT) {
    if (EXT && M.air && d.theta && (M.vmix != 0 || M.vmix_cd != 0) && d.L > 1)
      ISW_BATCH_L(d.L, LMAXK, fp64::vmix_heat_cell<LL>(M, d.h, d.theta, i));
  } else if (PH == PH_HF1) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_hf_edge<LL>(d.T, d.tr, 1, i / M.g.E, i % M.g.E));
  } else if (PH == PH_POST) {
    if (kind == 1) {
      if ((M.vmix != 0 || M.vmix_cd != 0) && d.L > 1) ISW_BATCH_L(d.L, LMAXK, fp64::vmix_edge<LL, EXT>(M, d.h, d.u, d.dt, i));
    } else {
      ISW_BATCH_L(d.L, LMAXK, fp64::tr_hf_edge<LL>(d.T, d.tr, 1, i / M.g.E, i % M.g.E));
    }
  } else if (PH == PH_P1) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_c1<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P2E) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_hf_edge<LL>(d.T, d.tr, 2, i / M.g.E, i % M.g.E));
  } else if (PH == PH_P2) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_c2<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P3E) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_a_edge<LL>(d.T, d.tr, i / M.g.E, i % M.g.E));
  } else if (PH == PH_P3) {
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_c3<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P4) {
    const int jj = i / M.g.N, c = i % M.g.N;
    ISW_BATCH_L(d.L, LMAXK, fp64::tr_p4<LL>(d.T, d.tr, jj, c));
    if (jj == 0)
      for (int l = 0; l < d.L; l++) d.Mm[(size_t)l * M.g.N + c] = d.tr.M1[(size_t)l * M.g.N + c];
  }
}

// The barotropic fast loop of stage `st` for every tiled stack (reference layers.cu:366-388, layers.py:168-175), one
// block per tile, all tiles of a group co-resident (cooperative launch). Same arithmetic as fp64::bt_eta_cell /
// bt_u_edge: the cell pass also forms each updated cell's Y = Gc (eta + gamma (eta - eta_prev)), the expression the
// reference's edge pass evaluates for each of an edge's two cells, so the edge pass reads two values per edge and no
// eta_prev is kept. Shared memory per edge: (l_e H_e, ubar) and (G, d_e) as 16-byte pairs; per cell its 8 edge slots
// as one 16-byte word. Exchange buffers (the owned values each round publishes, double-buffered by round parity):
// eta / eta_prev for the surface and ub2 / F for the barotropic wind (F, the layer fluxes, is not in use during the fast
// loop). The final barotropic wind and its accumulated sum go to ub and acc, which no round reads.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fast(const StackDesc *__restrict__ S, const TileRef *__restrict__ refs, int st,
                                                    int rounds, GridBarrier *bar, BatchStatus *status, long long timeout_ns,
                                                    int fault_block) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int cnt[2 * (FAST_KMAX + 1)];
  const TileRef tr = refs[blockIdx.x];
  const StackDesc &d = S[tr.s];
  const LayersDev &M = d.M;
  const TileSetDev &T = d.tiles;
  const int p = tr.p, k = T.k;
  const int c0 = T.cell_off[p], nc = T.cell_off[p + 1] - c0;
  const int e0 = T.edge_off[p], ne = T.edge_off[p + 1] - e0;
  const int eown = T.eown[p];
  const int *cells = T.cells + c0;
  const int *edges = T.edges + e0;
  double2 *EA = reinterpret_cast<double2 *>(smem);        // (l_e H_e, ubar)
  double2 *EB = EA + ne;                                   // (G, d_e)
  uint4 *cedge = reinterpret_cast<uint4 *>(EB + ne);       // 8 slots of +-(local edge + 1)
  double *acc = reinterpret_cast<double *>(cedge + nc);    // owned edges only
  double *eta = acc + eown;
  double *Y = eta + nc;
  double *area = Y + nc;
  double *gc = area + nc;
  short2 *eij = reinterpret_cast<short2 *>(gc + nc);
  const int skip = (int)blockIdx.x == fault_block;
  const int n = d.n[st];
  const double tau = d.tau[st], gam = M.div_damp;
  if (threadIdx.x <= k) {
    cnt[threadIdx.x] = T.ncnt[(size_t)p * (k + 1) + threadIdx.x];
    cnt[FAST_KMAX + 1 + threadIdx.x] = T.ecnt[(size_t)p * (k + 1) + threadIdx.x];
  }
  const uint4 *gcedge = reinterpret_cast<const uint4 *>(T.cedge) + c0;
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    const int gi = cells[c];
    eta[c] = M.eta0[gi];
    area[c] = T.aarea[c0 + c];
    gc[c] = M.Gc[gi];
    cedge[c] = gcedge[c];
  }
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const int ge = edges[e];
    EA[e] = make_double2(T.ale[e0 + e] * M.He[ge], M.ub0[ge]);
    EB[e] = make_double2(M.G[ge], T.ade[e0 + e]);
    if (e < eown) acc[e] = 0.0;
    eij[e] = make_short2(T.eIl[e0 + e], T.eJl[e0 + e]);
  }
  __syncthreads();
  const int nown = cnt[0];
  for (int r = 0; r < rounds; r++) {
    const int K = min(k, n - r * k);        // sub-steps of this stack in this round (<= 0: idle, barriers only)
    if (r > 0) {
      if (!grid_sync(bar, status, timeout_ns, skip)) return;
      if (K > 0) {                         // round r reads what round r - 1 published: buffer (r - 1) & 1
        const double *xe = ((r - 1) & 1) ? M.eta_prev : M.eta;
        const double *xu = ((r - 1) & 1) ? M.F : M.ub2;
        // only the halo: the owned cells and edges already hold exactly what was published
        for (int c = nown + threadIdx.x; c < nc; c += blockDim.x) eta[c] = xe[cells[c]];
        for (int e = eown + threadIdx.x; e < ne; e += blockDim.x) EA[e].y = xu[edges[e]];
      }
    }
    __syncthreads();
    for (int m = 1; m <= K; m++) {
      const int cn = cnt[K - m + 1];
      for (int c = threadIdx.x; c < cn; c += blockDim.x) {
        const double e0v = eta[c];
        const uint4 w = cedge[c];
        const int vs[6] = {(int16_t)(w.x & 0xffff), (int16_t)(w.x >> 16), (int16_t)(w.y & 0xffff), (int16_t)(w.y >> 16),
                           (int16_t)(w.z & 0xffff), (int16_t)(w.z >> 16)};
        double div = 0;
#pragma unroll
        for (int q = 0; q < 6; q++) {
          const int v = vs[q];
          if (v == 0) continue;
          const double2 pr = EA[(v > 0 ? v : -v) - 1];
          div += (v > 0 ? pr.x : -pr.x) * pr.y;
        }
        const double en = e0v - (tau * div) / area[c];
        eta[c] = en;
        Y[c] = gc[c] * (en + gam * (en - e0v));
      }
      __syncthreads();
      const int en = cnt[FAST_KMAX + 1 + K - m];
      for (int e = threadIdx.x; e < en; e += blockDim.x) {
        const double v = EA[e].y;
        const double2 gb = EB[e];
        const short2 ij = eij[e];
        if (e < eown) acc[e] += v;
        EA[e].y = v + tau * ((-(Y[ij.y] - Y[ij.x])) / gb.y + gb.x);
      }
      __syncthreads();
    }
    if (r + 1 < rounds && K > 0) {           // publish the owned values for the neighbours' next round: buffer r & 1
      double *xe = (r & 1) ? M.eta_prev : M.eta;
      double *xu = (r & 1) ? M.F : M.ub2;
      for (int c = threadIdx.x; c < nown; c += blockDim.x) xe[cells[c]] = eta[c];
      for (int e = threadIdx.x; e < eown; e += blockDim.x) xu[edges[e]] = EA[e].y;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < eown; e += blockDim.x) {
    M.ub[edges[e]] = EA[e].y;
    M.acc[edges[e]] = acc[e];
  }
}

// The grid-wide fast loop of stage `st` for the untiled FP64 stacks as ONE cooperative launch of co-resident blocks: each
// sub-step every block walks its share of the cell chunks (the eta pass), all blocks meet at the bounded grid barrier,
// walk the edge chunks (the ubar pass; with flux != 0 a stack's last sub-step also forms its layer fluxes, as PH_UF
// does) and meet again. The per-item arithmetic is PH_ETA's and PH_U's / PH_UF's, which otherwise take two launches
// per sub-step; the barrier's acquire makes every block's writes of one pass visible to the next pass.
template <int LMAXK, bool EXT>
__global__ void __launch_bounds__(THREADS) k_fast_grid(const StackDesc *__restrict__ S, const Sched sc, int st, int nsub,
                                                        int flux, GridBarrier *bar, BatchStatus *status, long long timeout_ns) {
  __shared__ __align__(16) unsigned char buf[sizeof(StackDesc)];
  const StackDesc &d = *reinterpret_cast<const StackDesc *>(buf);
  int cur = -1;
  auto select = [&](int s) {                 // the chunk's stack descriptor in shared memory (s is block-uniform)
    if (s == cur) return;
    __syncthreads();
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(S + s);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(buf);
    for (int w = threadIdx.x; w < (int)(sizeof(StackDesc) / 8); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    cur = s;
  };
  for (int j = 0; j < nsub; j++) {
    for (int c = blockIdx.x; c < sc.ncell; c += gridDim.x) {
      const Chunk ch = sc.cell[c];
      select(ch.s);
      const int i = ch.begin + (int)threadIdx.x;
      if (i < ch.end && !d.tiled && j < d.n[st]) {
        if (EXT && d.M.air) ISW_BATCH_L(d.L, LMAXK, fp64::af_muphi_cell<LL>(d.M, d.tau[st], i));
        else fp64::bt_eta_cell_y(d.M, d.tau[st], j, i);
      }
    }
    if (!grid_sync(bar, status, timeout_ns, 0)) return;
    for (int c = blockIdx.x; c < sc.nedge; c += gridDim.x) {
      const Chunk ch = sc.edge[c];
      select(ch.s);
      const int i = ch.begin + (int)threadIdx.x;
      if (i < ch.end && !d.tiled && j < d.n[st]) {
        if (EXT && d.M.air) {
          ISW_BATCH_L(d.L, LMAXK, fp64::af_u_edge<LL>(d.M, d.tau[st], i));
        } else {
          fp64::bt_u_edge_y<EXT>(d.M, d.tau[st], i);
          if (flux && j == d.n[st] - 1) fp64::flux_edge<EXT>(d.M, stage_args(d, st), d.M.acc[i], i);
        }
      }
    }
    if (!grid_sync(bar, status, timeout_ns, 0)) return;
  }
}

template <bool EXT>
const void *fast_grid_kernel_t(int lmax) {
  switch (lmax) {
    case 2: return (const void *)k_fast_grid<2, EXT>;
    case 3: return (const void *)k_fast_grid<3, EXT>;
    case 5: return (const void *)k_fast_grid<5, EXT>;
    default: return (const void *)k_fast_grid<8, EXT>;
  }
}

const void *fast_grid_kernel(int lmax, bool ext) { return ext ? fast_grid_kernel_t<true>(lmax) : fast_grid_kernel_t<false>(lmax); }

}  // namespace
}  // namespace isw

using namespace isw;

struct BatchSlot {
  bool used = false;
  isw_layers *layers = nullptr;
  isw_transport *tr = nullptr;
  double *h = nullptr, *u = nullptr, *Fm = nullptr, *M = nullptr, *M1 = nullptr;
  double *theta = nullptr;                  // air layers: the layers' potential temperature (L x N), else null
  int version = 0;                          // the layers' option version the descriptors were built from
  double *tracers[TRMAX] = {};
  int ntr = 0;
  double dt = 0;
  int nfast = 0;
};

struct FastGroup {
  int begin = 0, count = 0;
  size_t smem = 0;
  int rounds[3] = {0, 0, 0};
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
  Sched scf[2] = {};                          // chunk tables of the FP64 stacks [0] and the mixed ones [1]
  int lmax = 1, nstacks = 0, ntiles = 0, nsub[3] = {0, 0, 0}, kused = 0;
  std::vector<FastGroup> groups;              // cooperative launches of the fast loop (tiles [begin, begin + count))
  int any_nu4 = 0, any_vmix = 0, any_tr = 0, any_untiled = 0, any_air = 0;
  int any_ext = 0;                            // air or option stacks: the phase kernels with those branches
  int any_ob = 0;                             // a stack with the shelf's bed flags: their pass opens the step
  size_t fast_smem = 0;
  int fast_bps = 2;                           // tile blocks per SM: 2 (512 threads each) or 1 (1024 threads)
  GridBarrier *bar = nullptr;
  BatchStatus *status = nullptr;              // device status word (code + the mirror's device address)
  int *status_host = nullptr;                 // mapped pinned host mirror of the code, written by the failing kernel
  int tile_k = 8;
  int tiles_enabled = 1;
  int mixed = 0;                              // 1 when any stack is mixed: the tile kernels are then the mixed form's
  int tile_cells = 0;                         // packed layout's owned cells per tile (0: by blocks per SM)
  int force_bps = 0;                          // 0: choose; 1 or 2 tile blocks per SM
  int layout = 0;                             // 0: choose; 1 shared; 2 packed
  // per grid level: 0 follows the batch (default); 1 untiled; 2 packed tiles of about `cells` owned cells (0: the
  // batch's), exchange interval at most `k` (0: the batch's)
  struct LevelLayout {
    int mode = 0, cells = 0, k = 0;
  };
  std::map<int, LevelLayout> levels;
  bool pdl = true;                            // programmatic dependent launch between phase kernels
  bool fast_grid = false;                     // untiled stacks' sub-steps: one cooperative launch per stage (k_fast_grid)
  int untiled_form[2] = {0, 0};               // per form (FP64, mixed): any untiled stack
  size_t s_smem[2] = {0, 0};                  // per form: dynamic shared memory of the slow-tendency launch (staging)
  int grid_blocks[2] = {0, 0};                // per form: co-resident blocks of the cooperative grid-wide fast loop
  // pipelined steps: step n's dynamics beside step n-1's transport (two branches of one graph), Fm double-buffered.
  // desc[q] describes a step whose dynamics write Fm_q and whose transport reads it: Fm_0 the registered Fm, Fm_1 fm_alt
  bool pipeline = false, primed = false;
  int parity = 0;
  StackDesc *d_desc1 = nullptr;
  std::vector<void *> fm_alt;
  std::vector<std::pair<double *, size_t>> fm_pairs;  // (registered Fm, bytes) per stack, for the flush's copy-back
  cudaGraphExec_t pexec[6] = {};              // dynamics D_0, D_1; both branches DT_0, DT_1; transport T_0, T_1
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  const StackDesc *cur = nullptr;             // the descriptors the launches being queued use
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
constexpr int K_PROBE = FAST_KMAX;                       // the largest exchange interval considered

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

TileCache *tiles_for(isw_batch *b, const isw_grid *g, int P, int k);
int fitting_k(const TileSetHost &h, size_t budget, bool mixed, int threads);

// The largest exchange interval a tiling of g into P tiles fits in the budget, or 0 when no tiling can be built (a
// region too large or too scattered for the tiles' 16-bit local ids): the planners then leave the stack untiled.
int fitting_k_or_none(isw_batch *b, const isw_grid *g, int P, int kcap, size_t budget, int threads) {
  try {
    return fitting_k(tiles_for(b, g, P, std::min(K_PROBE, kcap))->host, budget, b->mixed == 1, threads);
  } catch (const Error &) {
    return 0;
  }
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
  std::vector<float> rde32(h.edges.size()), le32(h.edges.size()), rA32(h.cells.size());
  for (size_t q = 0; q < h.edges.size(); q++) { rde32[q] = (float)(1.0 / ade[q]); le32[q] = (float)ale[q]; }
  for (size_t q = 0; q < h.cells.size(); q++) rA32[q] = (float)(1.0 / aarea[q]);
  t.arde32 = dupload(c->allocs, rde32);
  t.ale32 = dupload(c->allocs, le32);
  t.arA32 = dupload(c->allocs, rA32);
  TileCache *out = c.get();
  b->tiles[key] = std::move(c);
  return out;
}

size_t smem_of(size_t nc, size_t ne, size_t nown, bool mixed) {
  return mixed ? tile_smem_bytes_mixed(nc, ne, nown) : tile_smem_bytes(nc, ne, nown);
}

// The largest k' <= the probe's k whose largest tile fits `budget` bytes of shared memory (0 if none).
// (mixed tiles also keep each thread's cells, edges and owned edges within the kernel's unrolled bounds)
int fitting_k(const TileSetHost &h, size_t budget, bool mixed, int threads) {
  for (int kk = h.k; kk >= 1; kk--) {
    size_t worst = 0;
    bool ok = true;
    for (int p = 0; p < h.P; p++) {
      const size_t nc = h.ncnt[(size_t)p * (h.k + 1) + kk], ne = h.ecnt[(size_t)p * (h.k + 1) + kk];
      worst = std::max(worst, smem_of(nc, ne, h.eown[p], mixed));
      if (mixed && (nc > (size_t)FAST_CMAX * threads || ne > (size_t)FAST_EMAX * threads ||
                    (size_t)h.eown[p] > (size_t)FAST_AMAX * threads))
        ok = false;
    }
    if (ok && worst <= budget) return kk;
  }
  return 0;
}

// Dynamic shared memory of the largest tile of a tile set.
size_t tiles_smem(const TileSetHost &h, bool mixed) {
  size_t worst = 0;
  for (int p = 0; p < h.P; p++)
    worst = std::max(worst, smem_of(h.cell_off[p + 1] - h.cell_off[p], h.edge_off[p + 1] - h.edge_off[p], h.eown[p], mixed));
  return worst;
}

int kernel_lmax(int L) { return L <= 2 ? 2 : L <= 3 ? 3 : L <= 5 ? 5 : 8; }

// The fast-loop tiling of the registered stacks. Two layouts, and the one with the larger exchange interval k wins:
//  - shared: one cooperative group over all stacks, each stack cut into tiles in proportion to its share of the cells,
//    filling the SMs (small batches: one member, a few members);
//  - packed: each stack cut into tiles of about tile_cells owned cells (a fixed size per grid, so tile sets are reused
//    as stacks come and go), the stacks packed in order into groups of at most SMs x blocks-per-SM tiles, one
//    cooperative launch per group and stage (large ensembles, serving).
// Stacks whose tiles would not fit in shared memory at all take the grid-wide sub-step kernels.
struct Tiling {
  int k = 0, bps = 2;                          // k: the smallest exchange interval over the stacks (the layout's score)
  std::vector<int> P;                          // tiles per slot (0: untiled)
  std::vector<int> K;                          // exchange interval per slot
  std::vector<int> group;                      // group per slot
};

int form_of(const BatchSlot &sl) { return sl.layers->d.precision == ISW_MIXED ? 1 : 0; }

// A batch holding stacks of both forms tiles the fast loop of its mixed stacks only (one tile kernel per batch); its
// FP64 stacks take the grid-wide sub-step kernels.
// Stacks with option branches: walls, the shelf (and its bed flags), per-cell buoyancy, the tide, the bottom's drag.
bool has_options(const isw::LayersDev &d) {
  return d.wall || d.ob || d.shelf > 0 || d.sig || d.tide || d.cbot || d.cd_bot > 0;
}

isw_batch::LevelLayout level_layout(const isw_batch *b, const BatchSlot &sl) {
  const auto it = b->levels.find(sl.layers->grid->n);
  return it == b->levels.end() ? isw_batch::LevelLayout{} : it->second;
}

bool tiles_form(const isw_batch *b, const BatchSlot &sl) {
  return sl.used && !sl.layers->d.air && !has_options(sl.layers->d) && form_of(sl) == b->mixed &&
         level_layout(b, sl).mode != 1;
}

Tiling plan_shared(isw_batch *b, int bps) {
  Tiling t;
  t.bps = bps;
  t.P.assign(b->slots.size(), 0);
  t.group.assign(b->slots.size(), 0);
  const size_t budget = bps == 2 ? SMEM_TWO : SMEM_ONE;
  const int slots = b->sms * bps;
  long long cells_total = 0;
  for (auto &sl : b->slots)
    if (tiles_form(b, sl)) cells_total += sl.layers->grid->d.N;
  int kmin = b->tile_k;
  bool any = false;
  for (size_t q = 0; q < b->slots.size(); q++) {
    const BatchSlot &sl = b->slots[q];
    if (!tiles_form(b, sl)) continue;
    const int N = sl.layers->grid->d.N;
    const int Pq = std::max(1, (int)((long long)slots * N / std::max(1LL, cells_total)));
    if (Pq * 16 > N) return Tiling{};          // tiles of at least 16 owned cells, for every stack
    const int kf = fitting_k_or_none(b, sl.layers->grid, Pq, b->tile_k, budget, bps == 2 ? 512 : 1024);
    if (kf == 0) return Tiling{};
    t.P[q] = Pq;
    kmin = std::min(kmin, kf);
    any = true;
  }
  t.k = any ? kmin : 0;
  t.K.assign(b->slots.size(), t.k);
  return t;
}

Tiling plan_packed(isw_batch *b, int bps) {
  Tiling t;
  t.bps = bps;
  t.P.assign(b->slots.size(), 0);
  t.K.assign(b->slots.size(), 0);
  t.group.assign(b->slots.size(), 0);
  const size_t budget = bps == 2 ? SMEM_TWO : SMEM_ONE;
  const int cap = b->sms * bps;
  const int cells_b = b->tile_cells > 0 ? b->tile_cells : (bps == 2 ? 384 : 768);
  int kmin = b->tile_k;
  bool any = false;
  for (size_t q = 0; q < b->slots.size(); q++) {
    const BatchSlot &sl = b->slots[q];
    if (!tiles_form(b, sl)) continue;
    const isw_batch::LevelLayout lv = level_layout(b, sl);       // the level's own tile size and interval, if set
    const int cells = lv.mode == 2 && lv.cells > 0 ? lv.cells : cells_b;
    const int kcap = lv.mode == 2 && lv.k > 0 ? std::min(lv.k, b->tile_k) : b->tile_k;
    const int N = sl.layers->grid->d.N;
    const int Pq = std::min(cap, std::max(1, (N + cells - 1) / cells));
    if (Pq * 16 > N) continue;
    const int kf = fitting_k_or_none(b, sl.layers->grid, Pq, kcap, budget, bps == 2 ? 512 : 1024);
    if (kf == 0) continue;
    t.P[q] = Pq;
    t.K[q] = kf;                               // each stack its own interval: a group's rounds follow its slowest
    kmin = std::min(kmin, kf);
    any = true;
  }
  if (!any) return Tiling{};
  t.k = kmin;
  int g = 0, fill = 0;
  for (size_t q = 0; q < b->slots.size(); q++) {
    if (t.P[q] == 0) continue;
    if (fill + t.P[q] > cap) { g++; fill = 0; }
    t.group[q] = g;
    fill += t.P[q];
  }
  return t;
}

void rebuild(isw_batch *b) {
  std::vector<StackDesc> desc;
  std::vector<Chunk> cell[2], edge[2], vert[2], rows[2], erows[2];      // per form: [0] FP64 stacks, [1] mixed
  std::vector<Chunk> wcell[2], wedge[2];                                // the sub-step passes' wide chunks
  int nsub[3] = {0, 0, 0};
  b->mixed = 0;
  for (auto &sl : b->slots)
    if (sl.used && form_of(sl) == 1) b->mixed = 1;
  int any_nu4 = 0, any_vmix = 0, any_tr = 0, any_untiled = 0, any_air = 0, any_ext = 0, any_ob = 0, lmax = 1;
  int untiled[2] = {0, 0};
  size_t s_smem[2] = {0, 0};
  const double cs[3] = {1.0 / 3.0, 1.0 / 2.0, 1.0};
  int used = 0;
  for (auto &sl : b->slots) used += sl.used ? 1 : 0;
  Tiling best;
  if (b->tiles_enabled && used > 0) {
    for (int bps = 2; bps >= 1; bps--) {
      if (b->force_bps && bps != b->force_bps) continue;
      if (b->layout != 2) {
        Tiling t = plan_shared(b, bps);
        if (t.k > best.k) best = t;
      }
      if (b->layout != 1) {
        Tiling t = plan_packed(b, bps);
        if (t.k > best.k || (b->layout == 2 && t.k > 0 && best.k == 0)) best = t;
      }
    }
  }
  const int kbest = best.k;
  const int ngroups = kbest > 0 ? 1 + *std::max_element(best.group.begin(), best.group.end()) : 0;
  std::vector<std::vector<TileRef>> grefs(ngroups);
  std::vector<size_t> gsmem(ngroups, 0);
  std::vector<std::array<int, 3>> gsub(ngroups, std::array<int, 3>{0, 0, 0});
  for (auto &sl : b->slots) {
    if (!sl.used) continue;
    StackDesc d;
    std::memset(&d, 0, sizeof(d));
    d.M = sl.layers->d;
    d.h = sl.h; d.u = sl.u; d.Fm = sl.Fm; d.Mm = sl.M;
    d.theta = sl.theta;
    if (d.M.air) any_air = 1;
    if (d.M.air || has_options(d.M)) any_ext = 1;
    if (d.M.ob) any_ob = 1;
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
    if (kbest > 0 && best.P[q] > 0) {
      TileCache *tc = tiles_for(b, sl.layers->grid, best.P[q], best.K[q]);
      const int g = best.group[q];
      d.tiled = 1;
      d.tiles = tc->dev;
      gsmem[g] = std::max(gsmem[g], tiles_smem(tc->host, b->mixed == 1));
      for (int p = 0; p < best.P[q]; p++) grefs[g].push_back(TileRef{s, p});
      for (int st = 0; st < 3; st++) gsub[g][st] = std::max(gsub[g][st], (d.n[st] + best.K[q] - 1) / best.K[q]);
    }
    if (!d.tiled) any_untiled = 1;
    {                                            // the mixed form's slow tendency stages its neighbour records when they fit
      // (measured: S 80.0 -> 76.2 us a level-6 member step in the mixed form; 97.4 -> 113.1 in FP64, whose 80-byte
      // records are staged about twice per block against the L1 hits of direct gathers, so FP64 gathers directly)
      const size_t need = (size_t)d.M.g.sMax * (size_t)d.L * sizeof(float4);
      d.s_stage = form_of(sl) == 1 && need <= S_STAGE_MAX ? 1 : 0;
      if (d.s_stage) s_smem[form_of(sl)] = std::max(s_smem[form_of(sl)], need);
    }
    auto chunks = [&](std::vector<Chunk> &v, int n, int w = THREADS) {
      for (int i = 0; i < n; i += w) v.push_back(Chunk{s, i, std::min(n, i + w)});
    };
    const int f = form_of(sl);
    if (!d.tiled) untiled[f] = 1;
    chunks(cell[f], d.M.g.N);
    chunks(edge[f], d.M.g.E);
    chunks(vert[f], d.M.g.NV);
    if (!d.tiled) {
      chunks(wcell[f], d.M.g.N, SUB_WC * THREADS);
      chunks(wedge[f], d.M.g.E, (f == 0 ? SUB_W_FP64 : SUB_W) * THREADS);
    }
    if (d.has_tr) chunks(rows[f], sl.ntr * d.M.g.N);       // (tracer, cell) pairs
    if (d.has_tr) chunks(erows[f], sl.ntr * d.M.g.E);      // (tracer, edge) pairs
    desc.push_back(d);
  }
  b->nstacks = (int)desc.size();
  cudaFree(b->d_desc);
  cudaFree(b->d_chunks);
  cudaFree(b->d_refs);
  b->d_desc = nullptr;
  b->d_chunks = nullptr;
  b->d_refs = nullptr;
  b->cur = nullptr;
  b->groups.clear();
  b->ntiles = 0;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  for (auto &x : b->pexec)
    if (x) {
      cudaGraphExecDestroy(x);
      x = nullptr;
    }
  cudaFree(b->d_desc1);
  b->d_desc1 = nullptr;
  for (void *q : b->fm_alt) cudaFree(q);
  b->fm_alt.clear();
  b->fm_pairs.clear();
  b->primed = false;
  b->parity = 0;
  b->dirty = false;
  if (desc.empty()) return;
  std::vector<Chunk> all;
  for (int f = 0; f < 2; f++) {
    all.insert(all.end(), cell[f].begin(), cell[f].end());
    all.insert(all.end(), edge[f].begin(), edge[f].end());
    all.insert(all.end(), vert[f].begin(), vert[f].end());
    all.insert(all.end(), rows[f].begin(), rows[f].end());
    all.insert(all.end(), erows[f].begin(), erows[f].end());
    all.insert(all.end(), wcell[f].begin(), wcell[f].end());
    all.insert(all.end(), wedge[f].begin(), wedge[f].end());
  }
  ISW_CUDA(cudaMalloc(&b->d_desc, sizeof(StackDesc) * desc.size()));
  ISW_CUDA(cudaMalloc(&b->d_chunks, sizeof(Chunk) * all.size()));
  ISW_CUDA(cudaMemcpy(b->d_chunks, all.data(), sizeof(Chunk) * all.size(), cudaMemcpyHostToDevice));
  std::vector<TileRef> refs;
  for (int g = 0; g < ngroups; g++) {
    FastGroup fg;
    fg.begin = (int)refs.size();
    fg.count = (int)grefs[g].size();
    fg.smem = gsmem[g];
    for (int st = 0; st < 3; st++) fg.rounds[st] = gsub[g][st];
    refs.insert(refs.end(), grefs[g].begin(), grefs[g].end());
    b->groups.push_back(fg);
  }
  b->fast_bps = best.bps;
  if (!refs.empty()) {                       // every tile block of a group must be resident at once (cooperative launch)
    const void *fn = b->mixed == 1 ? fast_kernel_mixed(best.bps)
                     : best.bps == 2 ? (const void *)k_fast<512, 2> : (const void *)k_fast<1024, 1>;
    size_t smax = 0;
    int cmax = 0;
    for (auto &fg : b->groups) { smax = std::max(smax, fg.smem); cmax = std::max(cmax, fg.count); }
    if (smax > 48 * 1024) ISW_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
    int per = 0;
    ISW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, best.bps == 2 ? 512 : 1024, smax));
    if ((long long)per * b->sms < cmax) {
      refs.clear();
      b->groups.clear();
      any_untiled = 1;
      for (auto &d : desc) d.tiled = 0;
      for (auto &sl : b->slots)
        if (sl.used) untiled[form_of(sl)] = 1;
    }
  }
  ISW_CUDA(cudaMemcpy(b->d_desc, desc.data(), sizeof(StackDesc) * desc.size(), cudaMemcpyHostToDevice));
  if (b->pipeline) {                         // the other parity's descriptors: the same stacks with a second Fm
    std::vector<StackDesc> desc1 = desc;
    for (auto &d : desc1) {
      const size_t bytes = sizeof(double) * (size_t)d.L * d.M.g.E;
      void *alt = nullptr;
      ISW_CUDA(cudaMalloc(&alt, bytes));
      ISW_CUDA(cudaMemset(alt, 0, bytes));
      b->fm_alt.push_back(alt);
      b->fm_pairs.emplace_back(d.Fm, bytes);
      d.Fm = (double *)alt;
      d.tr.Fm = (double *)alt;
    }
    ISW_CUDA(cudaMalloc(&b->d_desc1, sizeof(StackDesc) * desc1.size()));
    ISW_CUDA(cudaMemcpy(b->d_desc1, desc1.data(), sizeof(StackDesc) * desc1.size(), cudaMemcpyHostToDevice));
  }
  if (!refs.empty()) {
    ISW_CUDA(cudaMalloc(&b->d_refs, sizeof(TileRef) * refs.size()));
    ISW_CUDA(cudaMemcpy(b->d_refs, refs.data(), sizeof(TileRef) * refs.size(), cudaMemcpyHostToDevice));
  }
  const Chunk *base = b->d_chunks;
  for (int f = 0; f < 2; f++) {
    Sched &sc = b->scf[f];
    sc.status = b->status;
    sc.cell = base;
    sc.ncell = (int)cell[f].size();
    sc.edge = sc.cell + sc.ncell;
    sc.nedge = (int)edge[f].size();
    sc.vert = sc.edge + sc.nedge;
    sc.nvert = (int)vert[f].size();
    sc.rows = sc.vert + sc.nvert;
    sc.nrows = (int)rows[f].size();
    sc.erows = sc.rows + sc.nrows;
    sc.nerows = (int)erows[f].size();
    sc.wcell = sc.erows + sc.nerows;
    sc.nwcell = (int)wcell[f].size();
    sc.wedge = sc.wcell + sc.nwcell;
    sc.nwedge = (int)wedge[f].size();
    base = sc.wedge + sc.nwedge;
  }
  b->ntiles = (int)refs.size();
  size_t smax = 0;
  for (auto &fg : b->groups) smax = std::max(smax, fg.smem);
  b->fast_smem = smax;
  for (int st = 0; st < 3; st++) b->nsub[st] = nsub[st];
  b->kused = b->ntiles > 0 ? kbest : 0;
  b->any_nu4 = any_nu4;
  b->any_vmix = any_vmix;
  b->any_tr = any_tr;
  b->any_untiled = any_untiled;
  b->any_air = any_air;
  b->any_ext = any_ext;
  b->any_ob = any_ob;
  b->lmax = kernel_lmax(lmax);
  b->s_smem[0] = s_smem[0];
  b->s_smem[1] = s_smem[1];
  if (s_smem[0] > 48 * 1024)
    for (const void *fn : {(const void *)k_phase<PH_S, 2, false>, (const void *)k_phase<PH_S, 3, false>,
                           (const void *)k_phase<PH_S, 5, false>, (const void *)k_phase<PH_S, 8, false>,
                           (const void *)k_phase<PH_S, 2, true>, (const void *)k_phase<PH_S, 3, true>,
                           (const void *)k_phase<PH_S, 5, true>, (const void *)k_phase<PH_S, 8, true>})
      ISW_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_smem[0]));
  if (s_smem[1] > 48 * 1024) slow_phase_smem_mixed(s_smem[1]);
  for (int f = 0; f < 2; f++) {
    b->untiled_form[f] = untiled[f];
    b->grid_blocks[f] = 0;
    if (!untiled[f]) continue;
    int per = 0;
    const void *fn = f == 0 ? fast_grid_kernel(b->lmax, b->any_ext) : fast_grid_kernel_mixed();
    ISW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, THREADS, 0));
    b->grid_blocks[f] = std::max(1, per) * b->sms;
  }
}

// A phase over every stack: one kernel per precision form present (the FP64 stacks' first). pdl: the first of them is
// launched as a programmatic dependent of the kernel before it in the stream (never directly after a cooperative tile
// launch, which keeps plain stream order); a second one always is.
template <int PH>
void launch_phase(isw_batch *b, cudaStream_t st, int stage, int j, bool pdl = true) {
  bool first = true;
  for (int f = 0; f < 2; f++) {
    const Sched &sc = b->scf[f];
    const int nb = phase_blocks<PH>(sc);
    if (nb == 0) continue;
    if (!b->cur) fail(ISW_EINVAL, "batch: no stack descriptors selected for the launch");
    const bool p = (first ? pdl : true) && b->pdl;
    first = false;
    if (f == 1) {
      launch_phase_mixed(PH, b->lmax, nb, st, p, PH == PH_S ? b->s_smem[1] : 0, b->cur, sc, stage, j);
      continue;
    }
    const size_t smem = PH == PH_S ? b->s_smem[0] : 0;
    if (b->any_ext) {
      switch (b->lmax) {
        case 2: launch_phase_kernel(k_phase<PH, 2, true>, nb, st, p, smem, b->cur, sc, stage, j); break;
        case 3: launch_phase_kernel(k_phase<PH, 3, true>, nb, st, p, smem, b->cur, sc, stage, j); break;
        case 5: launch_phase_kernel(k_phase<PH, 5, true>, nb, st, p, smem, b->cur, sc, stage, j); break;
        default: launch_phase_kernel(k_phase<PH, 8, true>, nb, st, p, smem, b->cur, sc, stage, j); break;
      }
    } else {
      switch (b->lmax) {
        case 2: launch_phase_kernel(k_phase<PH, 2, false>, nb, st, p, smem, b->cur, sc, stage, j); break;
        case 3: launch_phase_kernel(k_phase<PH, 3, false>, nb, st, p, smem, b->cur, sc, stage, j); break;
        case 5: launch_phase_kernel(k_phase<PH, 5, false>, nb, st, p, smem, b->cur, sc, stage, j); break;
        default: launch_phase_kernel(k_phase<PH, 8, false>, nb, st, p, smem, b->cur, sc, stage, j); break;
      }
    }
  }
}

void launch_fast(isw_batch *b, cudaStream_t st, int stage, long long timeout_ns, int fault_block) {
  if (!b->groups.empty() && !b->cur) fail(ISW_EINVAL, "batch: no stack descriptors selected for the launch");
  for (const FastGroup &fg : b->groups) {
    if (fg.count == 0) continue;
    ISW_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(GridBarrier), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)fg.count);
    cfg.blockDim = dim3(b->fast_bps == 2 ? 512 : 1024);
    cfg.dynamicSmemBytes = fg.smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const TileRef *refs = b->d_refs + fg.begin;
    const StackDesc *desc = b->cur;
    const int rounds = fg.rounds[stage];
    if (b->mixed == 1)
      launch_fast_mixed(b->fast_bps, cfg, desc, refs, stage, rounds, b->bar, b->status, timeout_ns, fault_block);
    else if (b->fast_bps == 2)
      ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast<512, 2>, desc, refs, stage, rounds, b->bar, b->status, timeout_ns, fault_block));
    else
      ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast<1024, 1>, desc, refs, stage, rounds, b->bar, b->status, timeout_ns, fault_block));
    if (fault_block >= 0) break;             // the failure test runs the first group only
  }
}

// The untiled stacks' sub-steps of stage `stage` as one cooperative launch per form present (flux: the last sub-step
// also forms the layer fluxes, for a batch whose phase C only sums them).
void launch_fast_grid(isw_batch *b, cudaStream_t st, int stage, bool flux) {
  for (int f = 0; f < 2; f++) {
    const Sched &sc = b->scf[f];
    if (!b->untiled_form[f] || sc.ncell == 0) continue;
    if (!b->cur) fail(ISW_EINVAL, "batch: no stack descriptors selected for the launch");
    ISW_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(GridBarrier), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->grid_blocks[f]);
    cfg.blockDim = dim3(THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (f == 0) {
      const int fl = flux ? 1 : 0, ns = b->nsub[stage];
      long long to = DEFAULT_TIMEOUT_NS;
      void *args[] = {(void *)&b->cur, (void *)&sc, (void *)&stage, (void *)&ns, (void *)&fl, (void *)&b->bar,
                      (void *)&b->status, (void *)&to};
      ISW_CUDA(cudaLaunchKernelExC(&cfg, fast_grid_kernel(b->lmax, b->any_ext), args));
    } else
      launch_fast_grid_mixed(cfg, b->cur, sc, stage, b->nsub[stage], flux ? 1 : 0, b->bar, b->status, DEFAULT_TIMEOUT_NS);
  }
}

// The dynamics of one step (through the last stage's D). The first kernel and the first after a tile launch (or a
// memset) take plain stream order; the others are programmatic dependents of the kernel before them.
void enqueue_dyn(isw_batch *b, cudaStream_t st) {
  if (b->any_ob) launch_phase<PH_ONBED>(b, st, 0, 0, false);
  launch_phase<PH_INIT>(b, st, 0, 0, !b->any_ob ? false : true);
  if (b->any_nu4) {
    launch_phase<PH_LAPE1>(b, st, 0, 0);
    launch_phase<PH_LAPCV>(b, st, 0, 0);
    launch_phase<PH_LAPE2>(b, st, 0, 0);
  }
  for (int s = 0; s < 3; s++) {
    launch_phase<PH_A>(b, st, s, 0);
    launch_phase<PH_E>(b, st, s, 0);
    launch_phase<PH_S>(b, st, s, 0);
    const bool tiled = !b->groups.empty();
    launch_fast(b, st, s, DEFAULT_TIMEOUT_NS, -1);
    // no tiled stack: the layer fluxes are formed in the last grid-wide sub-step, once per edge, and C sums them
    const bool grid_loop = b->any_untiled && b->fast_grid;
    if (grid_loop) {
      launch_fast_grid(b, st, s, !tiled);
    } else if (b->any_untiled) {
      for (int j = 0; j < b->nsub[s]; j++) {
        launch_phase<PH_ETA>(b, st, s, j, !(tiled && j == 0));
        if (tiled) launch_phase<PH_U>(b, st, s, j);
        else launch_phase<PH_UF>(b, st, s, j);
      }
    }
    if (tiled) launch_phase<PH_C>(b, st, s, 0, b->any_untiled && !grid_loop);
    else launch_phase<PH_CS>(b, st, s, 0, !grid_loop);
    launch_phase<PH_D>(b, st, s, 0);
  }
}

// The transport passes after the stage-1 edge fluxes (P1 .. P4, M <- M1).
void enqueue_tr_tail(isw_batch *b, cudaStream_t st) {
  launch_phase<PH_P1>(b, st, 0, 0);
  launch_phase<PH_P2E>(b, st, 0, 0);
  launch_phase<PH_P2>(b, st, 0, 0);
  launch_phase<PH_P3E>(b, st, 0, 0);
  launch_phase<PH_P3>(b, st, 0, 0);
  launch_phase<PH_P4>(b, st, 0, 0);
}

// One step in the plain order: dynamics, then the interfacial stress with the transport's stage-1 edge fluxes, then
// the transport.
void enqueue(isw_batch *b, cudaStream_t st) {
  b->cur = b->d_desc;
  enqueue_dyn(b, st);
  if (b->any_air) {
    // air stacks: the interfacial stress's heat goes back to theta before the transport reads the tracers (theta is
    // one of them in the reference's world tick, world.py:291-301), so the stress, its heat and the stage-1 edge fluxes
    // are three passes here
    if (b->any_vmix) {
      launch_phase<PH_VMIX>(b, st, 0, 0);
      launch_phase<PH_VHEAT>(b, st, 0, 0);
    }
    if (b->any_tr) {
      launch_phase<PH_HF1>(b, st, 0, 0);
      enqueue_tr_tail(b, st);
    }
  } else {
    if (b->any_vmix || b->any_tr) launch_phase<PH_POST>(b, st, 0, 0);
    if (b->any_tr) enqueue_tr_tail(b, st);
  }
  ISW_CUDA(cudaGetLastError());
}

// Pipelined: the dynamics of the step described by `dyn` (with its interfacial stress) on `st`, and beside it on the
// side stream the transport of the step described by `tr` (the previous one); either may be null.
void enqueue_pipelined(isw_batch *b, cudaStream_t st, const StackDesc *dyn, const StackDesc *tr) {
  if (b->any_air) fail(ISW_EUNSUPPORTED, "batch: air stacks step in the plain order (the stress's heat precedes the transport)");
  const bool trans = tr && b->any_tr;
  if (trans && dyn) {
    ISW_CUDA(cudaEventRecord(b->ev_fork, st));
    ISW_CUDA(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
  }
  cudaStream_t ts = trans && dyn ? b->side : st;
  if (trans) {
    b->cur = tr;
    launch_phase<PH_HF1>(b, ts, 0, 0, false);
    enqueue_tr_tail(b, ts);
  }
  if (dyn) {
    b->cur = dyn;
    enqueue_dyn(b, st);
    if (b->any_vmix) launch_phase<PH_VMIX>(b, st, 0, 0);
  }
  if (trans && dyn) {
    ISW_CUDA(cudaEventRecord(b->ev_join, b->side));
    ISW_CUDA(cudaStreamWaitEvent(st, b->ev_join, 0));
  }
  ISW_CUDA(cudaGetLastError());
}

void prepare(isw_batch *b) {
  if (b->dirty) rebuild(b);
}

// Queue `body` on st: directly when st is capturing a graph of the caller's, else as a graph of our own (captured on
// the private stream the first time, cached in *exec).
template <class F>
void run_graph(isw_batch *b, cudaStream_t st, cudaGraphExec_t *exec, F body) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ISW_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {    // inside the caller's capture: queue the launches themselves
    body(st);
    return;
  }
  if (!*exec) {
    cudaGraph_t graph = nullptr;
    ISW_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    try {
      body(b->cap);
    } catch (...) {
      cudaStreamEndCapture(b->cap, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    ISW_CUDA(cudaStreamEndCapture(b->cap, &graph));
    const cudaError_t ie = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    ISW_CUDA(ie);
  }
  ISW_CUDA(cudaGraphLaunch(*exec, st));
}

const StackDesc *desc_of(isw_batch *b, int q) { return q == 0 ? b->d_desc : b->d_desc1; }

// Complete a pipelined batch: the last step's transport, and its Fm back into the registered arrays.
void flush(isw_batch *b, cudaStream_t st) {
  if (!b->pipeline || !b->primed) return;
  const int q = b->parity ^ 1;                // the last step's buffers
  if (b->any_tr) run_graph(b, st, &b->pexec[4 + q], [&](cudaStream_t s2) { enqueue_pipelined(b, s2, nullptr, desc_of(b, q)); });
  if (q == 1)
    for (size_t i = 0; i < b->fm_alt.size(); i++)
      ISW_CUDA(cudaMemcpyAsync(b->fm_pairs[i].first, b->fm_alt[i], b->fm_pairs[i].second, cudaMemcpyDeviceToDevice, st));
  b->primed = false;
}

// Flush a primed pipelined batch before its stacks or settings change (synchronising its private stream).
void settle(isw_batch *b) {
  if (b->pipeline && b->primed) {
    flush(b, b->cap);
    ISW_CUDA(cudaStreamSynchronize(b->cap));
  }
}

void step(isw_batch *b, cudaStream_t st) {
  for (auto &sl : b->slots)                  // an option set on a registered stack since: rebuild its descriptor
    if (sl.used && sl.version != sl.layers->version) {
      sl.version = sl.layers->version;
      b->dirty = true;
    }
  prepare(b);
  if (b->nstacks == 0) return;
  if (b->pipeline) {
    const int p = b->parity;
    const bool both = b->primed;
    run_graph(b, st, &b->pexec[both ? 2 + p : p],
              [&](cudaStream_t s2) { enqueue_pipelined(b, s2, desc_of(b, p), both ? desc_of(b, p ^ 1) : nullptr); });
    b->parity ^= 1;
    b->primed = true;
    return;
  }
  run_graph(b, st, &b->exec, [&](cudaStream_t s2) { enqueue(b, s2); });
}

}  // namespace

extern "C" {

int isw_batch_create(int device, isw_batch **out) {
  return guarded([&] {
    if (!out) fail(ISW_EINVAL, "batch: null output handle");
    ISW_CUDA(cudaSetDevice(device));
    isw_batch *b = new isw_batch();
    b->device = device;
    if (const char *e = std::getenv("ISW_NO_PDL")) b->pdl = e[0] != '1';   // diagnostics: plain stream order
    try {
      ISW_CUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device));
      ISW_CUDA(cudaMalloc(&b->bar, sizeof(GridBarrier)));
      ISW_CUDA(cudaMemset(b->bar, 0, sizeof(GridBarrier)));
      ISW_CUDA(cudaMalloc(&b->status, sizeof(BatchStatus)));
      ISW_CUDA(cudaHostAlloc((void **)&b->status_host, sizeof(int), cudaHostAllocMapped));
      *b->status_host = 0;
      BatchStatus init{0, 0, nullptr};
      ISW_CUDA(cudaHostGetDevicePointer((void **)&init.mirror, b->status_host, 0));
      ISW_CUDA(cudaMemcpy(b->status, &init, sizeof(BatchStatus), cudaMemcpyHostToDevice));
      ISW_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
      ISW_CUDA(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
      ISW_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
      ISW_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    } catch (...) {
      cudaFree(b->bar);
      cudaFree(b->status);
      if (b->status_host) cudaFreeHost(b->status_host);
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
  for (auto x : b->pexec)
    if (x) cudaGraphExecDestroy(x);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  cudaFree(b->d_desc1);
  for (void *q : b->fm_alt) cudaFree(q);
  cudaFree(b->d_desc);
  cudaFree(b->d_chunks);
  cudaFree(b->d_refs);
  cudaFree(b->bar);
  cudaFree(b->status);
  if (b->status_host) cudaFreeHost(b->status_host);
  for (auto &kv : b->tiles)
    for (void *p : kv.second->allocs) cudaFree(p);
  delete b;
  (void)cudaGetLastError();         // a failure while freeing must not surface in the caller's next call
  return ISW_OK;
}

namespace {

int batch_add(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *theta, double *M,
              double *M1, double *const *tracers, int ntr, double dt, int nfast, int *slot) {
  return guarded([&] {
    if (!b || !layers || !h || !u || !Fm || !slot) fail(ISW_EINVAL, "batch.add: null argument");
    if (layers->grid->device != b->device) fail(ISW_EINVAL, "batch.add: the stack is on another device");
    if (layers->d.air && !theta) fail(ISW_EINVAL, "batch.add: air layers need their theta (isw_batch_add_air)");
    if (!layers->d.air && theta) fail(ISW_EINVAL, "batch.add: theta is for air layers");
    if (has_options(layers->d) && layers->d.precision != ISW_FP64)
      fail(ISW_EUNSUPPORTED, "batch.add: the option branches step in the FP64 form");
    if (!(dt > 0) || !std::isfinite(dt) || nfast < 1) fail(ISW_EINVAL, "batch.add: dt must be positive and nfast >= 1");
    if (tr) {
      if (!M || !M1 || !tracers) fail(ISW_EINVAL, "batch.add: transport needs M, M1 and the tracers");
      if (ntr < 1 || ntr > tr->T) fail(ISW_EINVAL, "batch.add: ntr outside 1..tracers of the transport");
      if (tr->L != layers->d.L || tr->grid != layers->grid) fail(ISW_EINVAL, "batch.add: transport and layers differ in grid or L");
      if (tr->precision != layers->d.precision) fail(ISW_EINVAL, "batch.add: transport and layers differ in precision form");
    }
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    BatchSlot sl;
    sl.used = true;
    sl.layers = layers;
    sl.tr = tr;
    sl.h = h; sl.u = u; sl.Fm = Fm; sl.M = M; sl.M1 = M1;
    sl.theta = theta;
    sl.version = layers->version;
    if (layers->d.air && layers->d.nu4 != 0) layers->nu4dt = layers->d.nu4 * dt;   // the step's nabla^4 loss (exchange heat)
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

}  // namespace

int isw_batch_add(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *M, double *M1,
                  double *const *tracers, int ntr, double dt, int nfast, int *slot) {
  return batch_add(b, layers, tr, h, u, Fm, nullptr, M, M1, tracers, ntr, dt, nfast, slot);
}

int isw_batch_add_air(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *theta,
                      double *M, double *M1, double *const *tracers, int ntr, double dt, int nfast, int *slot) {
  return batch_add(b, layers, tr, h, u, Fm, theta, M, M1, tracers, ntr, dt, nfast, slot);
}

int isw_batch_remove(isw_batch *b, int slot) {
  return guarded([&] {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) fail(ISW_EINVAL, "batch.remove: no such slot");
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    b->slots[slot] = BatchSlot();
    b->dirty = true;
  });
}

int isw_batch_config(isw_batch *b, int tiles_enabled, int tile_k, int layout, int tile_cells, int blocks_per_sm) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.config: null handle");
    if (tile_k < 1 || tile_k > K_PROBE) fail(ISW_EINVAL, "batch.config: tile_k outside 1..8");
    if (layout < 0 || layout > 2) fail(ISW_EINVAL, "batch.config: layout must be 0 (choose), 1 (shared) or 2 (packed)");
    if (tile_cells != 0 && (tile_cells < 64 || tile_cells > 4096)) fail(ISW_EINVAL, "batch.config: tile_cells outside 64..4096");
    if (blocks_per_sm < 0 || blocks_per_sm > 2) fail(ISW_EINVAL, "batch.config: blocks_per_sm must be 0 (choose), 1 or 2");
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    b->tiles_enabled = tiles_enabled ? 1 : 0;
    b->tile_k = tile_k;
    b->layout = layout;
    b->tile_cells = tile_cells;
    b->force_bps = blocks_per_sm;
    b->dirty = true;
  });
}

int isw_batch_level_layout(isw_batch *b, int level, int mode, int tile_cells, int tile_k) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.level_layout: null handle");
    if (level < 0 || level > 12) fail(ISW_EINVAL, "batch.level_layout: level outside 0..12");
    if (mode < 0 || mode > 2) fail(ISW_EINVAL, "batch.level_layout: mode must be 0 (the batch's), 1 (untiled) or 2 (packed)");
    if (tile_cells != 0 && (tile_cells < 64 || tile_cells > 4096)) fail(ISW_EINVAL, "batch.level_layout: tile_cells outside 64..4096");
    if (tile_k < 0 || tile_k > K_PROBE) fail(ISW_EINVAL, "batch.level_layout: tile_k outside 0..8");
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    if (mode == 0) b->levels.erase(level);
    else b->levels[level] = isw_batch::LevelLayout{mode, tile_cells, tile_k};
    b->dirty = true;
  });
}

int isw_batch_grid_loop(isw_batch *b, int mode) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.grid_loop: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    if (mode != ISW_GRID_SPLIT && mode != ISW_GRID_PERSISTENT) fail(ISW_EINVAL, "batch.grid_loop: mode must be 0 or 1");
    b->fast_grid = mode == ISW_GRID_PERSISTENT;
    b->dirty = true;
  });
}

int isw_batch_info(isw_batch *b, int *stacks, int *tiles, int *tile_k, long long *smem_bytes, int *groups, int *blocks_per_sm) {
  return guarded([&] {
    if (!b || !stacks || !tiles || !tile_k || !smem_bytes || !groups || !blocks_per_sm) fail(ISW_EINVAL, "batch.info: null argument");
    ISW_CUDA(cudaSetDevice(b->device));
    prepare(b);
    *stacks = b->nstacks;
    *tiles = b->ntiles;
    *tile_k = b->ntiles > 0 ? b->kused : 0;
    *smem_bytes = (long long)b->fast_smem;
    *groups = (int)b->groups.size();
    *blocks_per_sm = b->ntiles > 0 ? b->fast_bps : 0;
  });
}

int isw_batch_step(isw_batch *b, void *stream) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.step: null handle");
    const int code = *(volatile int *)b->status_host;
    if (code == ISW_ETIMEOUT)
      fail(code, "batch.step: refused: an earlier step's grid barrier timed out, so the state is half-updated; restore "
                 "it and clear the status (isw_batch_status with reset) to step again");
    if (code != ISW_OK)
      fail(code, "batch.step: refused: an earlier step left a non-finite thickness; restore the state and clear the status "
                 "(isw_batch_status with reset) to step again");
    ISW_CUDA(cudaSetDevice(b->device));
    step(b, (cudaStream_t)stream);
  });
}

int isw_batch_pipeline(isw_batch *b, int on) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.pipeline: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    settle(b);
    b->pipeline = on != 0;
    b->dirty = true;
  });
}

int isw_batch_flush(isw_batch *b, void *stream) {
  return guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.flush: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    flush(b, (cudaStream_t)stream);
  });
}

int isw_batch_status(isw_batch *b, void *stream, int reset) {
  int out = ISW_OK;
  const int rc = guarded([&] {
    if (!b) fail(ISW_EINVAL, "batch.status: null handle");
    ISW_CUDA(cudaSetDevice(b->device));
    int st = 0;
    ISW_CUDA(cudaMemcpyAsync(&st, &b->status->code, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    ISW_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (reset) {
      ISW_CUDA(cudaMemset(&b->status->code, 0, sizeof(int)));
      ISW_CUDA(cudaDeviceSynchronize());
      *(volatile int *)b->status_host = 0;
    }
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
    if (b->groups.empty() || b->groups[0].rounds[2] < 2) fail(ISW_EUNSUPPORTED, "batch.fault_test: the last stage has no grid barrier");
    b->cur = b->d_desc;
    launch_fast(b, (cudaStream_t)stream, 2, timeout_ns, 0);
  });
}

}  // extern "C"
