// Flux-corrected tracer transport (reference src/insilica/transport.py:18-71 with kernels/fused.cu:122-241 and
// kernels/trisk.cu:48-59), plain FP64 form, and the Transport part of the C ABI.
//
// Rows y = tracer j * L + layer l, as the reference stacks them; row y's tracer values live in the caller's own array
// tracers[j] + l * N (no packed copy). Order 3 runs each RK stage as an edge pass (every 3rd-order edge flux computed
// once, for all layers of a (tracer, edge)) and a cell pass summing them in the reference's edge order, then the
// limited update: 7 launches against the reference's 8, bit-identical (transport_fp64.cuh).
//   HF1 / C1  stage-1 fluxes of psi; td (fused.cu:146-160) and p1 (fused.cu:163-186, frac 1/3) with the caller's M1
//   HF2 / C2  stage-2 fluxes of p1; p2 (frac 1/2)
//   A / C3    antidiffusive fluxes (fused.cu:189-194) and the Zalesak ratios (fused.cu:197-222)
//   P4        the limited update (fused.cu:225-241), written into the caller's tracer arrays
// Order 1 is td alone, copied out (the reference returns td): one cell pass (tr_p1).
#include <cstring>

#include "common.cuh"
#include "handles.cuh"

namespace isw {
namespace {

// reference trisk.cu:48-59
__global__ void __launch_bounds__(THREADS) k_mass(const GridDev g, int L, const double *__restrict__ M0, const double *__restrict__ Fm,
                                                  double *__restrict__ M1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.N * L) return;
  const int l = t / g.N, i = t - l * g.N;
  M1[(size_t)l * g.N + i] = fp64::mass_cell(g, M0, Fm + (size_t)l * g.E, l, i);
}

#define ISW_TR_L(LV, CALL)                              \
  do {                                                  \
    switch (LV) {                                       \
      case 1: { constexpr int LL = 1; CALL; } break;    \
      case 2: { constexpr int LL = 2; CALL; } break;    \
      case 3: { constexpr int LL = 3; CALL; } break;    \
      case 4: { constexpr int LL = 4; CALL; } break;    \
      case 5: { constexpr int LL = 5; CALL; } break;    \
      case 6: { constexpr int LL = 6; CALL; } break;    \
      case 7: { constexpr int LL = 7; CALL; } break;    \
      case 8: { constexpr int LL = 8; CALL; } break;    \
      default: break;                                   \
    }                                                   \
  } while (0)

// one thread per (tracer j, cell i), every layer of it
__global__ void __launch_bounds__(THREADS) k_p1(const TransportDev T, const TrArgs a, int ntr, int order) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * ntr) return;
  ISW_TR_L(a.L, fp64::tr_p1<LL>(T, a, order, false, t / T.g.N, t % T.g.N));
}

__global__ void __launch_bounds__(THREADS) k_hf(const TransportDev T, const TrArgs a, int ntr, int stage) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.E * ntr) return;
  ISW_TR_L(a.L, fp64::tr_hf_edge<LL>(T, a, stage, t / T.g.E, t % T.g.E));
}

__global__ void __launch_bounds__(THREADS) k_aflux(const TransportDev T, const TrArgs a, int ntr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.E * ntr) return;
  ISW_TR_L(a.L, fp64::tr_a_edge<LL>(T, a, t / T.g.E, t % T.g.E));
}

__global__ void __launch_bounds__(THREADS) k_c1(const TransportDev T, const TrArgs a, int ntr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * ntr) return;
  ISW_TR_L(a.L, fp64::tr_c1<LL>(T, a, t / T.g.N, t % T.g.N, false));
}

__global__ void __launch_bounds__(THREADS) k_c2(const TransportDev T, const TrArgs a, int ntr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * ntr) return;
  ISW_TR_L(a.L, fp64::tr_c2<LL>(T, a, t / T.g.N, t % T.g.N));
}

__global__ void __launch_bounds__(THREADS) k_c3(const TransportDev T, const TrArgs a, int ntr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * ntr) return;
  ISW_TR_L(a.L, fp64::tr_c3<LL>(T, a, t / T.g.N, t % T.g.N));
}

__global__ void __launch_bounds__(THREADS) k_p4(const TransportDev T, const TrArgs a, int ntr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * ntr) return;
  ISW_TR_L(a.L, fp64::tr_p4<LL>(T, a, t / T.g.N, t % T.g.N));
}

// order 1: td out
__global__ void __launch_bounds__(THREADS) k_td_out(const TransportDev T, const TrArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T.g.N * a.rows) return;
  const int y = t / T.g.N, i = t - y * T.g.N, l = y % a.L, j = y / a.L;
  a.tr[j][(size_t)l * T.g.N + i] = T.td[fx(j, T.g.N, i, a.L) + l];
}

}  // namespace
}  // namespace isw

using namespace isw;

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

double *talloc(isw_transport *t, size_t n) {
  void *p = nullptr;
  ISW_CUDA(cudaMalloc(&p, sizeof(double) * (n ? n : 1)));
  t->allocs.push_back(p);
  ISW_CUDA(cudaMemset(p, 0, sizeof(double) * (n ? n : 1)));
  return (double *)p;
}

}  // namespace

extern "C" {

int isw_transport_create(isw_grid *g, int L, double beta, int tracers, int precision, isw_transport **out) {
  return guarded([&] {
    if (!g || !out) fail(ISW_EINVAL, "transport: null grid or output handle");
    if (L < 1 || L > LMAX) fail(ISW_EINVAL, "transport: L must be in 1..8");
    if (tracers < 1 || tracers > TRMAX) fail(ISW_EINVAL, "transport: tracers must be in 1..16");
    if (precision != ISW_FP64 && precision != ISW_MIXED) fail(ISW_EINVAL, "transport: precision must be ISW_FP64 or ISW_MIXED");
    ISW_CUDA(cudaSetDevice(g->device));
    isw_transport *t = new isw_transport();
    t->grid = g;
    t->device = g->device;
    t->L = L;
    t->T = tracers;
    t->precision = precision;
    t->beta = beta;
    try {
      const size_t R = (size_t)lp_of(L) * tracers, N = g->d.N, E = g->d.E;   // layers side by side, padded to even
      t->d.g = g->d;
      t->d.td = talloc(t, R * N); t->d.p1 = talloc(t, R * N); t->d.p2 = talloc(t, R * N);
      t->d.Rp = talloc(t, R * N); t->d.Rm = talloc(t, R * N); t->d.A = talloc(t, R * E);
      if (precision == ISW_MIXED) {            // the batched step's mixed FCT: FP32 stage fields, fluxes and ratios
        auto f = [&](size_t n) { return reinterpret_cast<float *>(talloc(t, (n + 1) / 2)); };
        t->d.p1f = f(R * N); t->d.p2f = f(R * N); t->d.Af = f(R * E); t->d.Rpf = f(R * N); t->d.Rmf = f(R * N);
      }
    } catch (...) {
      for (void *p : t->allocs) cudaFree(p);
      delete t;
      throw;
    }
    *out = t;
  });
}

int isw_transport_destroy(isw_transport *t) {
  if (!t) return ISW_OK;
  cudaSetDevice(t->device);
  for (void *p : t->allocs) cudaFree(p);
  delete t;
  (void)cudaGetLastError();         // a failure while freeing must not surface in the caller's next call
  return ISW_OK;
}

int isw_transport_mass_after(isw_transport *t, const double *M0, const double *Fm, double *M1, void *stream) {
  return guarded([&] {
    if (!t || !M0 || !Fm || !M1) fail(ISW_EINVAL, "transport.mass_after: null argument");
    ISW_CUDA(cudaSetDevice(t->grid->device));
    const GridDev &g = t->d.g;
    k_mass<<<blocks_for((long long)g.N * t->L), THREADS, 0, (cudaStream_t)stream>>>(g, t->L, M0, Fm, M1);
    ISW_CUDA(cudaGetLastError());
  });
}

int isw_transport_step_many(isw_transport *t, const double *M0, const double *M1, const double *Fm, double *const *tracers, int ntr,
                            int order, void *stream) {
  return guarded([&] {
    if (!t || !M0 || !M1 || !Fm || !tracers) fail(ISW_EINVAL, "transport.step_many: null argument");
    if (ntr < 1 || ntr > t->T) fail(ISW_EINVAL, "transport.step_many: more tracers than the transport was built for");
    if (order != 1 && order != 3) fail(ISW_EINVAL, "transport.step_many: order must be 1 or 3");
    ISW_CUDA(cudaSetDevice(t->grid->device));
    TrArgs a;
    std::memset(&a, 0, sizeof(a));
    a.M0 = M0; a.M1 = const_cast<double *>(M1); a.Fm = Fm; a.L = t->L; a.rows = ntr * t->L; a.beta = t->beta;
    for (int j = 0; j < ntr; j++) {
      if (!tracers[j]) fail(ISW_EINVAL, "transport.step_many: null tracer");
      a.tr[j] = tracers[j];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = blocks_for((long long)t->d.g.N * ntr), ne = blocks_for((long long)t->d.g.E * ntr);
    if (order == 1) {
      k_p1<<<nb, THREADS, 0, st>>>(t->d, a, ntr, order);
      k_td_out<<<blocks_for((long long)t->d.g.N * a.rows), THREADS, 0, st>>>(t->d, a);
    } else {
      k_hf<<<ne, THREADS, 0, st>>>(t->d, a, ntr, 1);
      k_c1<<<nb, THREADS, 0, st>>>(t->d, a, ntr);
      k_hf<<<ne, THREADS, 0, st>>>(t->d, a, ntr, 2);
      k_c2<<<nb, THREADS, 0, st>>>(t->d, a, ntr);
      k_aflux<<<ne, THREADS, 0, st>>>(t->d, a, ntr);
      k_c3<<<nb, THREADS, 0, st>>>(t->d, a, ntr);
      k_p4<<<nb, THREADS, 0, st>>>(t->d, a, ntr);
    }
    ISW_CUDA(cudaGetLastError());
  });
}

}  // extern "C"
