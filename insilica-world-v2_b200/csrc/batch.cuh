// Definitions shared by the batched step's translation units (batch.cu: plain FP64 phases and the step's host side;
// batch_mixed.cu: the mixed form's phases, compiled with fused multiply-adds): the stack descriptor, chunk tables,
// tiles, the bounded grid barrier, the phase list.
#pragma once
#include <cuda/atomic>

#include "common.cuh"
#include "transport_fp64.cuh"

namespace isw {
namespace bt {

constexpr int FAST_KMAX = 8;                  // the largest exchange interval of the tiled fast loop
constexpr int FAST_CMAX = 4;                  // mixed tiles: cells per thread at most (nc <= FAST_CMAX x threads)
constexpr int FAST_EMAX = 8;                  // mixed tiles: edges per thread at most
constexpr int FAST_AMAX = 4;                  // mixed tiles: owned edges per thread at most (their sums in registers)

struct TileSetDev {
  int P, k;
  const int *cell_off, *edge_off, *cells, *edges, *ncnt, *ecnt, *eown;
  const int16_t *cedge, *eIl, *eJl;
  const double *ade, *ale, *aarea;            // d_e, l_e per local edge and the area per local cell, in local order
  const float *arde32, *ale32, *arA32;        // the mixed form's: 1 / d_e, l_e, 1 / area, in local order
};

struct StackDesc {
  LayersDev M;
  TransportDev T;
  TrArgs tr;                 // M0 = the stack's M, M1, Fm, tracers, L, rows, beta
  double *h, *u, *Fm, *Mm;
  double *theta;             // air layers: potential temperature (L x N); null for Boussinesq layers
  double dt;
  int L, has_tr, tiled;
  int s_stage;               // the slow tendency stages its blocks' neighbour records in shared memory
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

// The batch's status word on the device, and where a kernel that sets it also writes the code for the host: a mapped
// pinned host word, so that the next isw_batch_step can refuse to run without synchronising the stream.
struct BatchStatus {
  int code;
  int pad;
  volatile int *mirror;
};

// Record the first failure of a step (later ones keep the first code) and publish it to the host.
__device__ __forceinline__ void raise_status(BatchStatus *s, int code) {
  if (atomicCAS(&s->code, 0, code) == 0 && s->mirror) {
    *s->mirror = code;
    __threadfence_system();
  }
}

struct Sched {
  const Chunk *cell, *edge, *vert, *rows, *erows;   // rows: (tracer, cell) pairs; erows: (tracer, edge) pairs
  int ncell, nedge, nvert, nrows, nerows;
  const Chunk *wcell, *wedge;                       // the same in the sub-step passes' chunks (SUB_W... x THREADS)
  int nwcell, nwedge;
  BatchStatus *status;
};

// The step's result check: every layer of cell i must hold a finite thickness after the last stage, else the batch's
// status becomes ISW_ENOTFINITE (a NaN or Inf in a wind reaches the thicknesses through the layer fluxes in the same step).
__device__ __forceinline__ void check_finite_column(const double *__restrict__ h, int N, int L, int i, BatchStatus *s) {
  bool ok = true;
  for (int k = 0; k < L; k++) ok = ok && isfinite(h[(size_t)k * N + i]);
  if (!ok) raise_status(s, ISW_ENOTFINITE);
}

struct GridBarrier {
  unsigned count, gen;
};

__device__ __forceinline__ long long globaltimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Block-wide grid barrier with a bounded wait. Returns false once any block has recorded a failure.
__device__ inline bool grid_sync(GridBarrier *b, BatchStatus *status, long long timeout_ns, int skip_arrive) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(b->gen), cnt(b->count);
    cuda::atomic_ref<int, cuda::thread_scope_device> st(status->code);
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
            raise_status(status, ISW_ETIMEOUT);
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

#define ISW_BATCH_L(LV, LMAXK, ...)                                                             \
  do {                                                                                          \
    switch (LV) {                                                                               \
      case 1: { constexpr int LL = 1; __VA_ARGS__; } break;                                     \
      case 2: if (LMAXK >= 2) { constexpr int LL = 2 <= LMAXK ? 2 : 1; __VA_ARGS__; } break;    \
      case 3: if (LMAXK >= 3) { constexpr int LL = 3 <= LMAXK ? 3 : 1; __VA_ARGS__; } break;    \
      case 4: if (LMAXK >= 4) { constexpr int LL = 4 <= LMAXK ? 4 : 1; __VA_ARGS__; } break;    \
      case 5: if (LMAXK >= 5) { constexpr int LL = 5 <= LMAXK ? 5 : 1; __VA_ARGS__; } break;    \
      case 6: if (LMAXK >= 6) { constexpr int LL = 6 <= LMAXK ? 6 : 1; __VA_ARGS__; } break;    \
      case 7: if (LMAXK >= 7) { constexpr int LL = 7 <= LMAXK ? 7 : 1; __VA_ARGS__; } break;    \
      case 8: if (LMAXK >= 8) { constexpr int LL = 8 <= LMAXK ? 8 : 1; __VA_ARGS__; } break;    \
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

// The FCT step's passes: POST (edges: interfacial stress; (tracer, edge): stage-1 fluxes), P1 (cells: M1, td, p1),
// P2E (stage-2 fluxes), P2 (cells: p2), P3E (antidiffusive fluxes), P3 (cells: ratios), P4 (cells: limited update).
// A pipelined batch splits POST into VMIX (edges, the dynamics' last pass) and HF1 ((tracer, edge), the transport's first);
// a batch with air stacks runs VMIX, VHEAT (cells: the stress's heat back to theta) and HF1 in place of POST.
// PH_UF / PH_CS: the grid-wide edge sub-step that also forms the layer fluxes on a stack's last sub-step, and phase C
// summing them; used by batches with no tiled stack in place of PH_U / PH_C.
enum Phase { PH_INIT, PH_LAPE1, PH_LAPCV, PH_LAPE2, PH_A, PH_E, PH_S, PH_ETA, PH_U, PH_C, PH_D, PH_POST, PH_P2, PH_P3, PH_P4,
             PH_P1, PH_P2E, PH_P3E, PH_VMIX, PH_HF1, PH_UF, PH_CS, PH_VHEAT, PH_ONBED };

// Programmatic dependent launch between phase kernels: a phase kernel is launched while the previous one drains; it
// stages only constant data (its stack descriptor) before waiting for the previous grid's completion and memory
// (griddepcontrol.wait), and lets its own dependent launch at once (griddepcontrol.launch_dependents).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KA, class... A>
void launch_phase_kernel(void (*kern)(KA...), int nb, cudaStream_t st, bool pdl, size_t smem, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)nb);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  ISW_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}

// Domains of a phase, in block order: which chunk tables its blocks walk.
template <int PH>
struct Dom {
  static constexpr bool cell = PH == PH_INIT || PH == PH_LAPCV || PH == PH_A || PH == PH_ETA || PH == PH_C || PH == PH_D ||
                               PH == PH_CS || PH == PH_VHEAT || PH == PH_ONBED;
  static constexpr bool edge = PH == PH_INIT || PH == PH_LAPE1 || PH == PH_LAPE2 || PH == PH_E || PH == PH_S || PH == PH_U ||
                               PH == PH_D || PH == PH_POST || PH == PH_VMIX || PH == PH_UF;
  static constexpr bool vert = PH == PH_INIT || PH == PH_LAPCV || PH == PH_A;
  static constexpr bool rows = PH == PH_P1 || PH == PH_P2 || PH == PH_P3 || PH == PH_P4;
  static constexpr bool erows = PH == PH_POST || PH == PH_P2E || PH == PH_P3E || PH == PH_HF1;
  static constexpr bool wide = PH == PH_ETA || PH == PH_U || PH == PH_UF;   // cells / edges in the wide chunks
};

// Blocks of a phase over a schedule.
template <int PH>
inline int phase_blocks(const Sched &sc) {
  return (Dom<PH>::cell ? (Dom<PH>::wide ? sc.nwcell : sc.ncell) : 0) +
         (Dom<PH>::edge ? (Dom<PH>::wide ? sc.nwedge : sc.nedge) : 0) + (Dom<PH>::vert ? sc.nvert : 0) +
         (Dom<PH>::rows ? sc.nrows : 0) + (Dom<PH>::erows ? sc.nerows : 0);
}

// The chunk of block b of a phase and its kind (0 cell, 1 edge, 2 vertex, 3 (tracer, cell), 4 (tracer, edge)), or -1.
template <int PH>
__device__ __forceinline__ int phase_chunk(const Sched &sc, int b, Chunk &ch) {
  if (Dom<PH>::cell) {
    const int n = Dom<PH>::wide ? sc.nwcell : sc.ncell;
    if (b < n) { ch = (Dom<PH>::wide ? sc.wcell : sc.cell)[b]; return 0; }
    b -= n;
  }
  if (Dom<PH>::edge) {
    const int n = Dom<PH>::wide ? sc.nwedge : sc.nedge;
    if (b < n) { ch = (Dom<PH>::wide ? sc.wedge : sc.edge)[b]; return 1; }
    b -= n;
  }
  if (Dom<PH>::vert) { if (b < sc.nvert) { ch = sc.vert[b]; return 2; } b -= sc.nvert; }
  if (Dom<PH>::rows) { if (b < sc.nrows) { ch = sc.rows[b]; return 3; } b -= sc.nrows; }
  if (Dom<PH>::erows) { if (b < sc.nerows) { ch = sc.erows[b]; return 4; } }
  return -1;
}


constexpr size_t S_STAGE_MAX = 64 * 1024;   // the slow tendency's staged neighbour records: at most this per block

void launch_phase_mixed(int ph, int lmax, int nb, cudaStream_t st, bool pdl, size_t smem, const StackDesc *desc,
                        const Sched &sc, int stage, int j);
void slow_phase_smem_mixed(size_t bytes);
const void *fast_kernel_mixed(int bps);
const void *fast_grid_kernel_mixed();
void launch_fast_grid_mixed(const cudaLaunchConfig_t &cfg, const StackDesc *desc, const Sched &sc, int stage, int nsub,
                            int flux, GridBarrier *bar, BatchStatus *status, long long timeout_ns);
void launch_fast_mixed(int bps, const cudaLaunchConfig_t &cfg, const StackDesc *desc, const TileRef *refs, int stage, int rounds,
                       GridBarrier *bar, BatchStatus *status, long long timeout_ns, int fault_block);

}  // namespace bt
}  // namespace isw
