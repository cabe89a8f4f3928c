// The batched step's kernels for stacks in the mixed form (layers_mixed.cuh, transport_mixed.cuh): the same phase list,
// chunk tables and tiles as the plain FP64 kernels in batch.cu, compiled with fused multiply-adds (this file alone).
// The tile kernel runs the fast loop in deviation form (deta, dub in FP32, their FP64 sum acc) in shared memory.
#include "batch.cuh"
#include "layers_mixed.cuh"
#include "transport_mixed.cuh"

namespace isw {
namespace bt {
namespace {

__device__ __forceinline__ mixed::MStageArgs mstage_args(const StackDesc &d, int st) {
  const LayersDev &M = d.M;
  mixed::MStageArgs a;
  a.h0 = d.h;
  a.u0 = d.u;
  a.u0f = M.u32;
  a.hs = st == 0 ? d.h : st == 1 ? M.h1 : M.h2;
  a.us = st == 0 ? M.u32 : st == 1 ? M.u1f : M.u2f;
  a.hn = st == 0 ? M.h1 : st == 1 ? M.h2 : d.h;
  a.un = st == 2 ? d.u : nullptr;
  a.unf = st == 0 ? M.u1f : st == 1 ? M.u2f : nullptr;
  a.Fm = st == 2 ? d.Fm : nullptr;
  a.cdt = d.cdt[st];
  a.dt = d.dt;
  a.tau = (float)d.tau[st];
  a.inv_n = d.inv_n[st];
  a.n = d.n[st];
  return a;
}

// The grid-wide sub-step passes over a wide chunk: PH_ETA's cells (sub-step 0 item by item, as it also forms the slot
// coefficients), PH_U's / PH_UF's edges (PH_UF also forming the layer fluxes on the stack's last sub-step).
template <int PH>
__device__ __forceinline__ void substep_chunk(const StackDesc &d, int st, int j, const Chunk &ch) {
  if (d.tiled || j >= d.n[st]) return;
  const LayersDev &M = d.M;
  const float tau = (float)d.tau[st];
  const int first = ch.begin + (int)threadIdx.x;
  if (PH == PH_ETA) {
    if (j == 0)
      for (int i = first; i < ch.end; i += THREADS) mixed::bt_eta_cell(M, tau, 0, d.n[st], i);
    else
      mixed::bt_eta_cells<SUB_WC>(M, tau, j, d.n[st], first, ch.end);
  } else {
    mixed::bt_u_edges(M, tau, j, d.n[st], first, ch.end);
    if (PH == PH_UF && j == d.n[st] - 1) {
      const mixed::MStageArgs a = mstage_args(d, st);
      for (int i = first; i < ch.end; i += THREADS) mixed::flux_edge(M, a, M.acc[i], i);
    }
  }
}

template <int PH, int LMAXK>
__global__ void __launch_bounds__(THREADS) k_phase_m(const StackDesc *__restrict__ S, const Sched sc, int st, int j) {
  Chunk ch{0, 0, 0};
  const int kind = phase_chunk<PH>(sc, blockIdx.x, ch);
  if (kind < 0) return;
  const StackDesc &d = stage_desc(S, ch.s);
  pdl_wait();
  pdl_trigger();
  if (Dom<PH>::wide) {                       // the grid-wide sub-step passes: a wide chunk, SUB_W items a thread
    substep_chunk<PH>(d, st, j, ch);
    return;
  }
  const int i = ch.begin + (int)threadIdx.x;
  if (PH == PH_S && d.s_stage) {             // the block stages its rows' distinct neighbour records, then computes
    extern __shared__ __align__(16) float4 stg4[];
    const mixed::MStageArgs a = mstage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, mixed::stage_pk4<LL>(d.M, ch.begin / THREADS, stg4));
    __syncthreads();
    if (i < ch.end) ISW_BATCH_L(d.L, LMAXK, (mixed::slow_edge<LL, true>(d.M, a.us, a.cdt, i, stg4)));
    return;
  }
  if (i >= ch.end) return;
  const LayersDev &M = d.M;
  if (PH == PH_INIT) {
    if (kind == 0) {
      ISW_BATCH_L(d.L, LMAXK, fp64::eta0_cell<LL>(M, d.h, i));
      if (M.nu4 != 0) ISW_BATCH_L(d.L, LMAXK, (mixed::div_cell<LL, double>(M, d.u, i)));
    } else if (kind == 1) {
      ISW_BATCH_L(d.L, LMAXK, mixed::ubar0_edge<LL>(M, d.h, d.u, i));
    } else if (M.nu4 != 0) {
      ISW_BATCH_L(d.L, LMAXK, (mixed::curl_vertex<LL, double>(M, d.u, i)));
    }
  } else if (PH == PH_LAPE1 || PH == PH_LAPE2) {
    if (M.nu4 != 0) ISW_BATCH_L(d.L, LMAXK, mixed::lap_edge<LL>(M, PH == PH_LAPE1 ? M.L1f : M.L2f, i));
  } else if (PH == PH_LAPCV) {
    if (M.nu4 != 0) {
      if (kind == 0) ISW_BATCH_L(d.L, LMAXK, (mixed::div_cell<LL, float>(M, M.L1f, i)));
      else ISW_BATCH_L(d.L, LMAXK, (mixed::curl_vertex<LL, float>(M, M.L1f, i)));
    }
  } else if (PH == PH_A) {
    const mixed::MStageArgs a = mstage_args(d, st);
    if (kind == 0) ISW_BATCH_L(d.L, LMAXK, mixed::bern_cell<LL>(M, a.hs, a.us, i));
    else ISW_BATCH_L(d.L, LMAXK, mixed::pv_vertex<LL>(M, a.hs, a.us, i));
  } else if (PH == PH_E) {
    const mixed::MStageArgs a = mstage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, mixed::edge_hq<LL>(M, a.hs, a.us, i));
  } else if (PH == PH_S) {
    const mixed::MStageArgs a = mstage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, mixed::slow_edge<LL>(M, a.us, a.cdt, i));
  } else if (PH == PH_C) {
    const mixed::MStageArgs a = mstage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, mixed::scale_cell<LL>(M, a, i));
  } else if (PH == PH_CS) {
    const mixed::MStageArgs a = mstage_args(d, st);
    ISW_BATCH_L(d.L, LMAXK, mixed::scale_sum_cell<LL>(M, a, i));
  } else if (PH == PH_D) {
    const mixed::MStageArgs a = mstage_args(d, st);
    if (kind == 0) {
      ISW_BATCH_L(d.L, LMAXK, mixed::h_cell<LL>(M, a, i));
      if (st == 2) check_finite_column(d.h, M.g.N, d.L, i, sc.status);
    } else {
      ISW_BATCH_L(d.L, LMAXK, mixed::u_edge<LL>(M, a, i));
    }
  } else if (PH == PH_VMIX) {
    if ((M.vmix != 0 || M.vmix_cd != 0) && d.L > 1) ISW_BATCH_L(d.L, LMAXK, fp64::vmix_edge<LL, false>(M, d.h, d.u, d.dt, i));
  } else if (PH == PH_HF1) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_hf_edge<LL>(d.T, d.tr, 1, i / M.g.E, i % M.g.E));
  } else if (PH == PH_POST) {
    if (kind == 1) {
      if ((M.vmix != 0 || M.vmix_cd != 0) && d.L > 1) ISW_BATCH_L(d.L, LMAXK, fp64::vmix_edge<LL, false>(M, d.h, d.u, d.dt, i));
    } else {
      ISW_BATCH_L(d.L, LMAXK, mixed::tr_hf_edge<LL>(d.T, d.tr, 1, i / M.g.E, i % M.g.E));
    }
  } else if (PH == PH_P1) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_c1<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P2E) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_hf_edge<LL>(d.T, d.tr, 2, i / M.g.E, i % M.g.E));
  } else if (PH == PH_P2) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_c2<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P3E) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_a_edge<LL>(d.T, d.tr, i / M.g.E, i % M.g.E));
  } else if (PH == PH_P3) {
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_c3<LL>(d.T, d.tr, i / M.g.N, i % M.g.N));
  } else if (PH == PH_P4) {
    const int jj = i / M.g.N, c = i % M.g.N;
    ISW_BATCH_L(d.L, LMAXK, mixed::tr_p4<LL>(d.T, d.tr, jj, c));
    if (jj == 0)
      for (int l = 0; l < d.L; l++) d.Mm[(size_t)l * M.g.N + c] = d.tr.M1[(size_t)l * M.g.N + c];
  }
}

// The fast loop of stage `st` over every tiled stack in the mixed form (the tile scheme of batch.cu's k_fast). Shared
// memory, FP32 arrays: per cell deta, Y = Gc (deta + gamma (deta - deta_prev)), 1/area, Gc, c0 = sum sign l_e H_e ubar0
// and its 8 edge slots (16 bytes); per edge dub, fl = l_e H_e dub (what the cell pass sums: one float per gathered
// edge), l_e H_e, G', 1/d_e and its two local cells. A thread's edges are always e = tid + j NT, so the FP64 sub-step
// sum acc of its owned edges (j < FAST_AMAX) stays in registers. Exchange buffers xeta[r & 1] and xdub[r & 1]; the
// final dub and acc go to dub and acc, which no round reads. The host keeps nc <= FAST_CMAX NT, ne <= FAST_EMAX NT and
// eown <= FAST_AMAX NT.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fast_m(const StackDesc *__restrict__ S, const TileRef *__restrict__ refs, int st,
                                                      int rounds, GridBarrier *bar, BatchStatus *status, long long timeout_ns,
                                                      int fault_block) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int cnt[2 * (FAST_KMAX + 1)];
  const TileRef tr = refs[blockIdx.x];
  const StackDesc &d = S[tr.s];
  const LayersDev &M = d.M;
  const TileSetDev &T = d.tiles;
  const int p = tr.p, k = T.k;
  const int c0i = T.cell_off[p], nc = T.cell_off[p + 1] - c0i;
  const int e0 = T.edge_off[p], ne = T.edge_off[p + 1] - e0;
  const int eown = T.eown[p];
  const int *cells = T.cells + c0i;
  const int *edges = T.edges + e0;
  uint4 *cedge = reinterpret_cast<uint4 *>(smem);
  float *deta = reinterpret_cast<float *>(cedge + nc);
  float *Y = deta + nc;
  float *rA = Y + nc;
  float *gc = rA + nc;
  float *cz = gc + nc;
  float *dub = cz + nc;
  float *fl = dub + ne;
  float *lh = fl + ne;
  float *G = lh + ne;
  float *rde = G + ne;
  short2 *eij = reinterpret_cast<short2 *>(rde + ne);
  const int skip = (int)blockIdx.x == fault_block;
  const int n = d.n[st];
  const float tau = (float)d.tau[st], gam = (float)M.div_damp;
  const int t = threadIdx.x;
  if (t <= k) {
    cnt[t] = T.ncnt[(size_t)p * (k + 1) + t];
    cnt[FAST_KMAX + 1 + t] = T.ecnt[(size_t)p * (k + 1) + t];
  }
  double accr[FAST_AMAX];
#pragma unroll
  for (int j = 0; j < FAST_AMAX; j++) accr[j] = 0.0;
  const uint4 *gcedge = reinterpret_cast<const uint4 *>(T.cedge) + c0i;
  for (int c = t; c < nc; c += NT) {
    deta[c] = 0.f;
    rA[c] = T.arA32[c0i + c];
    gc[c] = M.Gc32[cells[c]];
    cedge[c] = gcedge[c];
  }
  for (int e = t; e < ne; e += NT) {
    const int ge = edges[e];
    const float l = T.ale32[e0 + e] * M.He32[ge];
    lh[e] = l;
    fl[e] = l * (float)M.ub0[ge];          // ubar0's flux for the c0 pass below, then zero
    G[e] = M.G32[ge];
    rde[e] = T.arde32[e0 + e];
    eij[e] = make_short2(T.eIl[e0 + e], T.eJl[e0 + e]);
  }
  __syncthreads();
  for (int c = t; c < nc; c += NT) {
    const uint4 w = cedge[c];
    const int vs[6] = {(int16_t)(w.x & 0xffff), (int16_t)(w.x >> 16), (int16_t)(w.y & 0xffff), (int16_t)(w.y >> 16),
                       (int16_t)(w.z & 0xffff), (int16_t)(w.z >> 16)};
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int v = vs[q];
      if (v == 0) continue;
      const float f = fl[(v > 0 ? v : -v) - 1];
      s += v > 0 ? f : -f;
    }
    cz[c] = s;
  }
  __syncthreads();
  for (int e = t; e < ne; e += NT) {
    dub[e] = 0.f;
    fl[e] = 0.f;
  }
  const int nown = cnt[0];
  for (int r = 0; r < rounds; r++) {
    const int K = min(k, n - r * k);
    if (r > 0) {
      if (!grid_sync(bar, status, timeout_ns, skip)) return;
      if (K > 0) {
        const float *xe = M.xeta[(r - 1) & 1];
        const float *xu = M.xdub[(r - 1) & 1];
        for (int c = nown + t; c < nc; c += NT) deta[c] = xe[cells[c]];
        for (int e = eown + t; e < ne; e += NT) {
          const float v = xu[edges[e]];
          dub[e] = v;
          fl[e] = lh[e] * v;
        }
      }
    }
    __syncthreads();
    for (int m = 1; m <= K; m++) {
      const int cn = cnt[K - m + 1];
#pragma unroll
      for (int j = 0; j < FAST_CMAX; j++) {
        const int c = t + j * NT;
        if (c < cn) {
          const float d0 = deta[c];
          const uint4 w = cedge[c];
          const int vs[6] = {(int16_t)(w.x & 0xffff), (int16_t)(w.x >> 16), (int16_t)(w.y & 0xffff), (int16_t)(w.y >> 16),
                             (int16_t)(w.z & 0xffff), (int16_t)(w.z >> 16)};
          float div = cz[c];
#pragma unroll
          for (int q = 0; q < 6; q++) {
            const int v = vs[q];
            if (v == 0) continue;
            const float f = fl[(v > 0 ? v : -v) - 1];
            div += v > 0 ? f : -f;
          }
          const float dn = d0 - tau * div * rA[c];
          deta[c] = dn;
          Y[c] = gc[c] * (dn + gam * (dn - d0));
        }
      }
      __syncthreads();
      const int en = cnt[FAST_KMAX + 1 + K - m];
#pragma unroll
      for (int j = 0; j < FAST_EMAX; j++) {
        const int e = t + j * NT;
        if (e < en) {
          const float v = dub[e];
          const short2 ij = eij[e];
          if (j < FAST_AMAX && e < eown) accr[j < FAST_AMAX ? j : 0] += (double)v;
          const float nv = v + tau * (G[e] - (Y[ij.y] - Y[ij.x]) * rde[e]);
          dub[e] = nv;
          fl[e] = lh[e] * nv;
        }
      }
      __syncthreads();
    }
    if (r + 1 < rounds && K > 0) {
      float *xe = M.xeta[r & 1];
      float *xu = M.xdub[r & 1];
      for (int c = t; c < nown; c += NT) xe[cells[c]] = deta[c];
      for (int e = t; e < eown; e += NT) xu[edges[e]] = dub[e];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < FAST_AMAX; j++) {
    const int e = t + j * NT;
    if (e < eown) {
      M.dub[edges[e]] = dub[e];
      M.acc[edges[e]] = accr[j];
    }
  }
}

template <int PH>
void launch_m(int lmax, int nb, cudaStream_t st, bool pdl, size_t smem, const StackDesc *desc, const Sched &sc, int stage,
              int j) {
  switch (lmax) {
    case 2: launch_phase_kernel(k_phase_m<PH, 2>, nb, st, pdl, smem, desc, sc, stage, j); break;
    case 3: launch_phase_kernel(k_phase_m<PH, 3>, nb, st, pdl, smem, desc, sc, stage, j); break;
    case 5: launch_phase_kernel(k_phase_m<PH, 5>, nb, st, pdl, smem, desc, sc, stage, j); break;
    default: launch_phase_kernel(k_phase_m<PH, 8>, nb, st, pdl, smem, desc, sc, stage, j); break;
  }
}

}  // namespace

void slow_phase_smem_mixed(size_t bytes) {
  for (const void *fn : {(const void *)k_phase_m<PH_S, 2>, (const void *)k_phase_m<PH_S, 3>, (const void *)k_phase_m<PH_S, 5>,
                         (const void *)k_phase_m<PH_S, 8>})
    ISW_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

void launch_phase_mixed(int ph, int lmax, int nb, cudaStream_t st, bool pdl, size_t smem, const StackDesc *desc,
                        const Sched &sc, int stage, int j) {
  switch (ph) {
    case PH_INIT: launch_m<PH_INIT>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_LAPE1: launch_m<PH_LAPE1>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_LAPCV: launch_m<PH_LAPCV>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_LAPE2: launch_m<PH_LAPE2>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_A: launch_m<PH_A>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_E: launch_m<PH_E>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_S: launch_m<PH_S>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_ETA: launch_m<PH_ETA>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_U: launch_m<PH_U>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_C: launch_m<PH_C>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_UF: launch_m<PH_UF>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_CS: launch_m<PH_CS>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_D: launch_m<PH_D>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_POST: launch_m<PH_POST>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P2: launch_m<PH_P2>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P3: launch_m<PH_P3>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P4: launch_m<PH_P4>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P1: launch_m<PH_P1>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P2E: launch_m<PH_P2E>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_P3E: launch_m<PH_P3E>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_VMIX: launch_m<PH_VMIX>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    case PH_HF1: launch_m<PH_HF1>(lmax, nb, st, pdl, smem, desc, sc, stage, j); break;
    default: break;
  }
}

namespace {

// The grid-wide fast loop of stage `st` for the untiled mixed stacks as one cooperative launch (batch.cu's k_fast_grid
// with the mixed form's per-item arithmetic: PH_ETA's and PH_U's / PH_UF's of k_phase_m).
__global__ void __launch_bounds__(THREADS) k_fast_grid_m(const StackDesc *__restrict__ S, const Sched sc, int st, int nsub,
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
      if (i < ch.end && !d.tiled && j < d.n[st]) mixed::bt_eta_cell(d.M, (float)d.tau[st], j, d.n[st], i);
    }
    if (!grid_sync(bar, status, timeout_ns, 0)) return;
    for (int c = blockIdx.x; c < sc.nedge; c += gridDim.x) {
      const Chunk ch = sc.edge[c];
      select(ch.s);
      const int i = ch.begin + (int)threadIdx.x;
      if (i < ch.end && !d.tiled && j < d.n[st]) {
        mixed::bt_u_edge(d.M, (float)d.tau[st], j, d.n[st], i);
        if (flux && j == d.n[st] - 1) mixed::flux_edge(d.M, mstage_args(d, st), d.M.acc[i], i);
      }
    }
    if (!grid_sync(bar, status, timeout_ns, 0)) return;
  }
}

}  // namespace

const void *fast_grid_kernel_mixed() { return (const void *)k_fast_grid_m; }

void launch_fast_grid_mixed(const cudaLaunchConfig_t &cfg, const StackDesc *desc, const Sched &sc, int stage, int nsub,
                            int flux, GridBarrier *bar, BatchStatus *status, long long timeout_ns) {
  ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast_grid_m, desc, sc, stage, nsub, flux, bar, status, timeout_ns));
}

const void *fast_kernel_mixed(int bps) {
  return bps == 2 ? (const void *)k_fast_m<512, 2> : (const void *)k_fast_m<1024, 1>;
}

void launch_fast_mixed(int bps, const cudaLaunchConfig_t &cfg, const StackDesc *desc, const TileRef *refs, int stage, int rounds,
                       GridBarrier *bar, BatchStatus *status, long long timeout_ns, int fault_block) {
  if (bps == 2)
    ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast_m<512, 2>, desc, refs, stage, rounds, bar, status, timeout_ns, fault_block));
  else
    ISW_CUDA(cudaLaunchKernelEx(&cfg, k_fast_m<1024, 1>, desc, refs, stage, rounds, bar, status, timeout_ns, fault_block));
}

}  // namespace bt
}  // namespace isw
