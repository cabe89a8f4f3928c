// The stacked-layer step (reference src/insilica/layers.py:35-212): kernels over the phase functions of layers_fp64.cuh,
// the step's launch sequence, the CUDA-graph cache for direct calls, and the Layers part of the C ABI.
//
// Launch sequence of one step: init, [lap cv, lap e] x 2 if nu4, then per stage: A, E, S, n x (eta, ubar), C, D; then
// vmix if set. 21 + 2 sum_s n_s launches (95 at nfast = 20), against the reference's 35 + 2 sum_s n_s (+6 with nu4).
// A direct call (stream not capturing) replays a cached CUDA graph of the whole step: one launch from the host.
#include <cmath>
#include <cstring>
#include <list>
#include <sstream>

#include "common.cuh"
#include "handles.cuh"
#include "layers_air.cuh"
#include "layers_fp64.cuh"
#include "layers_xch.cuh"

namespace isw {
namespace {

template <int L>
__global__ void __launch_bounds__(THREADS) k_init(const LayersDev M, const double *__restrict__ h, const double *__restrict__ u) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::eta0_cell<L>(M, h, t);
  else if (t < M.g.N + M.g.E) fp64::ubar0_edge<L>(M, h, u, t - M.g.N);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_lap_cv(const LayersDev M, const double *__restrict__ u) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::div_cell<L>(M, u, t);
  else if (t < M.g.N + M.g.NV) fp64::curl_vertex<L>(M, u, t - M.g.N);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_lap_e(const LayersDev M, double *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::lap_edge<L>(M, out, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_stage_a(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::bern_cell<L>(M, a.hs, a.us, t);
  else if (t < M.g.N + M.g.NV) fp64::pv_vertex<L>(M, a.hs, a.us, t - M.g.N);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_stage_e(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::edge_hq<L>(M, a.hs, a.us, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_stage_s(const LayersDev M, const StageArgs a, const double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::slow_edge<L>(M, a.us, a.cdt, t, theta);
}

// ---- air layers ----
template <int L>
__global__ void __launch_bounds__(THREADS) k_air_stiff(const LayersDev M, const double *__restrict__ h, const double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::air_stiff_cell<L>(M, h, theta, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_air_gfast(const LayersDev M, const double *__restrict__ h, const double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::air_gfast_cell<L>(M, h, theta, t);
}

// stage A for air: B and pibar, the PV pass, and the fast state's masses
template <int L>
__global__ void __launch_bounds__(THREADS) k_air_a(const LayersDev M, const StageArgs a, const double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) {
    fp64::air_bern_cell<L>(M, a.hs, a.us, theta, t);
    fp64::air_fast_init_cell<L>(M, a.h0, t);
  } else if (t < M.g.N + M.g.NV) {
    fp64::pv_vertex<L>(M, a.hs, a.us, t - M.g.N);
  }
}

// stage E for air: the edge records and the fast state's winds
template <int L>
__global__ void __launch_bounds__(THREADS) k_air_e(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) {
    fp64::edge_hq<L>(M, a.hs, a.us, t);
    fp64::air_fast_init_edge<L>(M, a.u0, t);
  }
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_af_muphi(const LayersDev M, double tau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::af_muphi_cell<L>(M, tau, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_af_u(const LayersDev M, double tau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::af_u_edge<L>(M, tau, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_air_c(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::air_scale_cell<L>(M, a, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_air_d(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::h_cell<L>(M, a, t);
  else if (t < M.g.N + M.g.E) fp64::air_u_edge<L>(M, a, t - M.g.N);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_onbed(const LayersDev M, const double *__restrict__ h) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::onbed_cell<L>(M, h, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_xch_cell(const LayersDev M, const double *__restrict__ wx, double *h, double *Mm,
                                                      double *psi, int seq) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::xch_cell<L>(M, wx, h, Mm, psi, seq, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_xch_edge(const LayersDev M, const double *__restrict__ wx, double *u, double *diss,
                                                      const double *lap4, double nu4dt, double hthin) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::xch_edge<L>(M, wx, M.hold, u, diss, lap4, nu4dt, hthin, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_vmix_heat(const LayersDev M, const double *__restrict__ h, double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::vmix_heat_cell<L>(M, h, theta, t);
}

// The heating kernel of the layers' kernel table as the world calls it after the sea coupling (reference
// world.py:317-318 with kernels/layers.cu:596-621): the caller's per-edge dissipation and constants.
template <int L>
__global__ void __launch_bounds__(THREADS) k_heat(const GridDev g, const double *__restrict__ h, const double *__restrict__ diss,
                                                  double grav, double cp, double kap, double p0, double *__restrict__ theta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < g.N) fp64::heat_column<L>(g, h, diss, grav, cp, kap, p0, theta, t);
}

// rows of an edge field zeroed on the wall edges (reference kernels/layers.cu:495-499, lay_mask)
__global__ void __launch_bounds__(THREADS) k_wall_mask(const double *__restrict__ wall, int E, int rows, double *__restrict__ a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E || wall[e] != 0) return;
  for (int k = 0; k < rows; k++) a[(size_t)k * E + e] = 0;
}

__global__ void __launch_bounds__(THREADS) k_bt_eta(const LayersDev M, double tau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::bt_eta_cell(M, tau, t);
}

__global__ void __launch_bounds__(THREADS) k_bt_u(const LayersDev M, double tau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::bt_u_edge(M, tau, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_stage_c(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::scale_cell<L>(M, a, t);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_stage_d(const LayersDev M, const StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.N) fp64::h_cell<L>(M, a, t);
  else if (t < M.g.N + M.g.E) fp64::u_edge<L>(M, a, t - M.g.N);
}

template <int L>
__global__ void __launch_bounds__(THREADS) k_vmix(const LayersDev M, const double *__restrict__ h, double *__restrict__ u, double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M.g.E) fp64::vmix_edge<L>(M, h, u, dt, t);
}

// max over cells of g sum_k h_k: per-block maxima, then one block over them (values are >= 0 for a valid state;
// NaN propagates as NaN through fmax's operand order below only if every value is NaN, so a separate flag counts NaNs)
__global__ void __launch_bounds__(THREADS) k_colmax(const LayersDev M, const double *__restrict__ h, double *out, int *nonfinite) {
  __shared__ double s[THREADS];
  double m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M.g.N; i += gridDim.x * blockDim.x) {
    double c = 0;
    for (int k = 0; k < M.L; k++) c += h[(size_t)k * M.g.N + i];
    const double v = c * M.Gc[i];
    if (!isfinite(v)) atomicAdd(nonfinite, 1);
    else m = fmax(m, v);
  }
  s[threadIdx.x] = m;
  __syncthreads();
  for (int w = THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void k_max_reduce(const double *in, int n, double *out) {
  __shared__ double s[THREADS];
  double m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, in[i]);
  s[threadIdx.x] = m;
  __syncthreads();
  for (int w = THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

#define ISW_DISPATCH_L(L, CALL)                      \
  switch (L) {                                        \
    case 1: { constexpr int LL = 1; CALL; } break;    \
    case 2: { constexpr int LL = 2; CALL; } break;    \
    case 3: { constexpr int LL = 3; CALL; } break;    \
    case 4: { constexpr int LL = 4; CALL; } break;    \
    case 5: { constexpr int LL = 5; CALL; } break;    \
    case 6: { constexpr int LL = 6; CALL; } break;    \
    case 7: { constexpr int LL = 7; CALL; } break;    \
    case 8: { constexpr int LL = 8; CALL; } break;    \
    default: fail(ISW_EINVAL, "layers: L outside 1..8"); \
  }

}  // namespace
}  // namespace isw

using namespace isw;

namespace {

constexpr size_t GRAPH_CACHE = 8;

double *dalloc(isw_layers *s, size_t n) {
  void *p = nullptr;
  ISW_CUDA(cudaMalloc(&p, sizeof(double) * (n ? n : 1)));
  s->allocs.push_back(p);
  ISW_CUDA(cudaMemset(p, 0, sizeof(double) * (n ? n : 1)));
  return (double *)p;
}

template <class T>
T *talloc_t(isw_layers *s, size_t n) {
  void *p = nullptr;
  ISW_CUDA(cudaMalloc(&p, sizeof(T) * (n ? n : 1)));
  s->allocs.push_back(p);
  ISW_CUDA(cudaMemset(p, 0, sizeof(T) * (n ? n : 1)));
  return (T *)p;
}

// The step's kernels in order on `st` (reference layers.py:185-212, Boussinesq branch).
void enqueue_step(isw_layers *s, double *h, double *u, double *Fm, double dt, int nfast, cudaStream_t st) {
  const LayersDev &M = s->d;
  const GridDev &g = M.g;
  const int L = M.L;
  const int N = g.N, E = g.E, NV = g.NV;
  if (M.ob) ISW_DISPATCH_L(L, (k_onbed<LL><<<blocks_for(N), THREADS, 0, st>>>(M, h)));
  ISW_DISPATCH_L(L, (k_init<LL><<<blocks_for(N + E), THREADS, 0, st>>>(M, h, u)));
  if (M.nu4 != 0) {
    ISW_DISPATCH_L(L, (k_lap_cv<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, u)));
    ISW_DISPATCH_L(L, (k_lap_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, M.L1)));
    ISW_DISPATCH_L(L, (k_lap_cv<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, M.L1)));
    ISW_DISPATCH_L(L, (k_lap_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, M.L2)));
  }
  const double cs[3] = {1.0 / 3.0, 1.0 / 2.0, 1.0};
  for (int st_i = 0; st_i < 3; st_i++) {
    const double c = cs[st_i];
    StageArgs a;
    a.h0 = h;
    a.u0 = u;
    a.hs = st_i == 0 ? h : st_i == 1 ? M.h1 : M.h2;
    a.us = st_i == 0 ? u : st_i == 1 ? M.u1 : M.u2;
    a.hn = st_i == 0 ? M.h1 : st_i == 1 ? M.h2 : h;
    a.un = st_i == 0 ? M.u1 : st_i == 1 ? M.u2 : u;
    a.Fm = st_i == 2 ? Fm : nullptr;
    a.cdt = c * dt;
    a.dt = dt;
    const double cn = std::ceil(c * nfast);
    a.n = cn > 1 ? (int)cn : 1;
    a.tau = c * dt / a.n;
    a.inv_n = 1.0 / a.n;
    ISW_DISPATCH_L(L, (k_stage_a<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, a)));
    ISW_DISPATCH_L(L, (k_stage_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, a)));
    ISW_DISPATCH_L(L, (k_stage_s<LL><<<blocks_for(E), THREADS, 0, st>>>(M, a, nullptr)));
    for (int j = 0; j < a.n; j++) {
      k_bt_eta<<<blocks_for(N), THREADS, 0, st>>>(M, a.tau);
      k_bt_u<<<blocks_for(E), THREADS, 0, st>>>(M, a.tau);
    }
    ISW_DISPATCH_L(L, (k_stage_c<LL><<<blocks_for(N), THREADS, 0, st>>>(M, a)));
    ISW_DISPATCH_L(L, (k_stage_d<LL><<<blocks_for(N + E), THREADS, 0, st>>>(M, a)));
  }
  if ((M.vmix != 0 || M.vmix_cd != 0) && L > 1)
    ISW_DISPATCH_L(L, (k_vmix<LL><<<blocks_for(E), THREADS, 0, st>>>(M, h, u, dt)));
  ISW_CUDA(cudaGetLastError());
}

// One step of air layers in order on `st` (reference layers.py:185-206 with _stage's air branch, :134-136, 152-166):
// air_stiff, the nabla^4 passes, per stage A (air_bern + PV + fast masses), E (+ fast winds), S (+ pibar grad theta),
// n x (af_muphi, af_u), C (af_flux + lay_scale), D (lay_h, u = uf, Fm); then vmix and its heat.
void enqueue_step_air(isw_layers *s, double *h, double *u, double *Fm, double *theta, double dt, int nfast, cudaStream_t st) {
  const LayersDev &M = s->d;
  const GridDev &g = M.g;
  const int L = M.L;
  const int N = g.N, E = g.E, NV = g.NV;
  ISW_DISPATCH_L(L, (k_air_stiff<LL><<<blocks_for(N), THREADS, 0, st>>>(M, h, theta)));
  if (M.nu4 != 0) {
    ISW_DISPATCH_L(L, (k_lap_cv<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, u)));
    ISW_DISPATCH_L(L, (k_lap_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, M.L1)));
    ISW_DISPATCH_L(L, (k_lap_cv<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, M.L1)));
    ISW_DISPATCH_L(L, (k_lap_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, M.L2)));
  }
  const double cs[3] = {1.0 / 3.0, 1.0 / 2.0, 1.0};
  for (int st_i = 0; st_i < 3; st_i++) {
    const double c = cs[st_i];
    StageArgs a;
    a.h0 = h;
    a.u0 = u;
    a.hs = st_i == 0 ? h : st_i == 1 ? M.h1 : M.h2;
    a.us = st_i == 0 ? u : st_i == 1 ? M.u1 : M.u2;
    a.hn = st_i == 0 ? M.h1 : st_i == 1 ? M.h2 : h;
    a.un = st_i == 0 ? M.u1 : st_i == 1 ? M.u2 : u;
    a.Fm = st_i == 2 ? Fm : nullptr;
    a.cdt = c * dt;
    a.dt = dt;
    const double cn = std::ceil(c * nfast);
    a.n = cn > 1 ? (int)cn : 1;
    a.tau = c * dt / a.n;
    a.inv_n = 1.0 / a.n;
    ISW_DISPATCH_L(L, (k_air_a<LL><<<blocks_for(N + NV), THREADS, 0, st>>>(M, a, theta)));
    ISW_DISPATCH_L(L, (k_air_e<LL><<<blocks_for(E), THREADS, 0, st>>>(M, a)));
    ISW_DISPATCH_L(L, (k_stage_s<LL><<<blocks_for(E), THREADS, 0, st>>>(M, a, theta)));
    for (int j = 0; j < a.n; j++) {
      ISW_DISPATCH_L(L, (k_af_muphi<LL><<<blocks_for(N), THREADS, 0, st>>>(M, a.tau)));
      ISW_DISPATCH_L(L, (k_af_u<LL><<<blocks_for(E), THREADS, 0, st>>>(M, a.tau)));
    }
    ISW_DISPATCH_L(L, (k_air_c<LL><<<blocks_for(N), THREADS, 0, st>>>(M, a)));
    ISW_DISPATCH_L(L, (k_air_d<LL><<<blocks_for(N + E), THREADS, 0, st>>>(M, a)));
  }
  if ((M.vmix != 0 || M.vmix_cd != 0) && L > 1) {
    ISW_DISPATCH_L(L, (k_vmix<LL><<<blocks_for(E), THREADS, 0, st>>>(M, h, u, dt)));
    ISW_DISPATCH_L(L, (k_vmix_heat<LL><<<blocks_for(N), THREADS, 0, st>>>(M, h, theta)));
  }
  ISW_CUDA(cudaGetLastError());
}

isw_layers *layers_create(isw_grid *g, const isw_layers_params *p) {
  if (!g || !p) fail(ISW_EINVAL, "layers: null grid or parameters");
  if (p->L < 1 || p->L > LMAX) fail(ISW_EINVAL, "layers: L must be in 1..8");
  if (p->L > 1 && !p->gprime) fail(ISW_EINVAL, "layers: gprime needs L - 1 values");
  if (p->precision != ISW_FP64 && p->precision != ISW_MIXED) fail(ISW_EINVAL, "layers: precision must be ISW_FP64 or ISW_MIXED");
  if (p->air && p->precision != ISW_FP64) fail(ISW_EUNSUPPORTED, "layers: air layers run in the FP64 form only");
  if (p->air && !(p->cp > 0 && p->kappa > 0 && p->rd > 0 && p->p0 > 0)) fail(ISW_EINVAL, "layers: air constants must be positive");
  if ((p->wall || p->shelf != 0 || p->shelf_bed) && p->precision != ISW_FP64)
    fail(ISW_EUNSUPPORTED, "layers: walls and the shelf run in the FP64 form only");
  if (p->wall && p->air) fail(ISW_EINVAL, "layers: walls are for Boussinesq layers");
  if (!(p->shelf >= 0)) fail(ISW_EINVAL, "layers: shelf must be >= 0");
  ISW_CUDA(cudaSetDevice(g->device));
  isw_layers *s = new isw_layers();
  s->grid = g;
  s->device = g->device;
  try {
    LayersDev &d = s->d;
    std::memset(&d, 0, sizeof(d));
    d.g = g->d;
    d.L = p->L;
    d.precision = p->precision;
    d.grav = p->grav;
    d.nu4 = p->nu4;
    d.floor_ = p->floor_;
    d.div_damp = p->div_damp;
    d.thin = p->thin;
    d.vmix = p->vmix;
    d.vmix_cd = p->vmix_cd;
    for (int k = 0; k < LMAX; k++) {
      d.gp[k] = (p->L > 1 && k < p->L - 1) ? p->gprime[k] : 0.0;
      d.drag[k] = (p->drag && k < p->L) ? p->drag[k] : 0.0;
      d.stress[k] = (p->stress && k < p->L) ? p->stress[k] : 0.0;
    }
    const int N = g->d.N, E = g->d.E, NV = g->d.NV, L = p->L;
    double *b = dalloc(s, N);
    if (p->b) ISW_CUDA(cudaMemcpy(b, p->b, sizeof(double) * N, cudaMemcpyHostToDevice));
    d.b = b;
    std::vector<double> hv(NV);
    ISW_CUDA(cudaMemcpy(hv.data(), g->d.fV, sizeof(double) * NV, cudaMemcpyDeviceToHost));
    for (int v = 0; v < NV; v++) hv[v] = hv[v] * p->rotation;       // self.fV = dg.fV * rotation (layers.py:62)
    double *fV = dalloc(s, NV);
    ISW_CUDA(cudaMemcpy(fV, hv.data(), sizeof(double) * NV, cudaMemcpyHostToDevice));
    d.fV = fV;
    std::vector<double> gc(N, p->grav);
    double *Gc = dalloc(s, N);
    ISW_CUDA(cudaMemcpy(Gc, gc.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    d.Gc = Gc;
    d.B = dalloc(s, (size_t)L * N); d.q = dalloc(s, (size_t)L * NV); d.Tp = dalloc(s, (size_t)L * E);
    d.F = dalloc(s, (size_t)L * E); d.scale = dalloc(s, (size_t)L * N);
    d.G = dalloc(s, E); d.He = dalloc(s, E); d.ubs = dalloc(s, E); d.ub0 = dalloc(s, E); d.ub = dalloc(s, E); d.acc = dalloc(s, E);
    d.eta0 = dalloc(s, N); d.eta = dalloc(s, N); d.eta_prev = dalloc(s, N);
    d.h1 = dalloc(s, (size_t)L * N); d.h2 = dalloc(s, (size_t)L * N); d.u1 = dalloc(s, (size_t)L * E); d.u2 = dalloc(s, (size_t)L * E);
    d.D1 = dalloc(s, (size_t)L * N); d.Z1 = dalloc(s, (size_t)L * NV); d.L1 = dalloc(s, (size_t)L * E); d.L2 = dalloc(s, (size_t)L * E);
    d.hedge = dalloc(s, (size_t)L * E); d.diss = dalloc(s, E); d.pk = dalloc(s, (size_t)pk_stride(L) * E);
    d.ub2 = dalloc(s, E);
    d.cw = dalloc(s, (size_t)N * 6);
    d.hold = dalloc(s, (size_t)L * N);
    d.thin_wind = p->thin_wind;
    s->percall = p->percall != 0;
    if (p->wall) {
      double *w = dalloc(s, E);
      ISW_CUDA(cudaMemcpy(w, p->wall, sizeof(double) * E, cudaMemcpyHostToDevice));
      d.wall = w;
    }
    d.shelf = p->shelf;
    if (p->shelf_bed && p->shelf > 0) d.ob = dalloc(s, (size_t)L * N);
    if (p->air) {
      d.air = 1;
      d.cpa = p->cp; d.kap = p->kappa; d.rda = p->rd; d.p0 = p->p0;
      d.S = dalloc(s, (size_t)L * N); d.pibar = dalloc(s, (size_t)L * N); d.muf = dalloc(s, (size_t)L * N);
      d.phi = dalloc(s, (size_t)L * N); d.uf = dalloc(s, (size_t)L * E); d.accL = dalloc(s, (size_t)L * E);
    }
    if (p->precision == ISW_MIXED) {
      auto f = [&](size_t n) { return talloc_t<float>(s, n); };
      d.u32 = f((size_t)L * E); d.u1f = f((size_t)L * E); d.u2f = f((size_t)L * E);
      d.D1f = f((size_t)L * N); d.Z1f = f((size_t)L * NV); d.L1f = f((size_t)L * E); d.L2f = f((size_t)L * E);
      d.q32 = f((size_t)L * NV); d.Tp32 = f((size_t)L * E); d.G32 = f(E); d.He32 = f(E); d.ubs32 = f(E);
      d.dub = f(E); d.deta = f(N); d.deprev = f(N); d.cw32 = f((size_t)N * 8);
      d.Gr32 = talloc_t<float2>(s, E);
      d.F32 = f((size_t)L * E); d.scale32 = f((size_t)L * N);
      d.wsum = dalloc(s, N);
      d.xeta[0] = f(N); d.xeta[1] = f(N); d.xdub[0] = f(E); d.xdub[1] = f(E);
      d.pk4 = talloc_t<float4>(s, (size_t)L * E);
      std::vector<float> gc32(N, (float)p->grav);
      d.Gc32 = f(N);
      ISW_CUDA(cudaMemcpy(d.Gc32, gc32.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
    }
    s->colmax_blocks = blocks_for(N) < 1024 ? blocks_for(N) : 1024;
    d.red = dalloc(s, s->colmax_blocks + 1);
    void *nf = nullptr;
    ISW_CUDA(cudaMalloc(&nf, sizeof(int)));
    s->allocs.push_back(nf);
    s->nonfinite = (int *)nf;
    ISW_CUDA(cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking));
  } catch (...) {
    for (void *q : s->allocs) cudaFree(q);
    delete s;
    throw;
  }
  return s;
}

void layers_destroy(isw_layers *s) {
  cudaSetDevice(s->device);
  if (s->solo) isw_batch_destroy(s->solo);
  for (auto &e : s->graphs) cudaGraphExecDestroy(e.exec);
  if (s->cap) cudaStreamDestroy(s->cap);
  for (void *p : s->allocs) cudaFree(p);
  delete s;
  (void)cudaGetLastError();         // a failure while freeing must not surface in the caller's next call
}

// A step call by call through a private batch holding this one stack (rebuilt when the arrays, dt or nfast change): the
// tiled fast loop and one graph per step. The mixed form always steps this way; the FP64 form does when the stack has
// no air and no option branches, with bit-identical results.
void layers_step_solo(isw_layers *s, double *h, double *u, double *Fm, double dt, int nfast, cudaStream_t st) {
  auto ok = [](int rc) { if (rc != ISW_OK) fail(rc, isw_last_error()); };
  if (!s->solo) ok(isw_batch_create(s->grid->device, &s->solo));
  if (!Fm) {
    if (!s->solo_Fm) s->solo_Fm = dalloc(s, (size_t)s->d.L * s->d.g.E);
    Fm = s->solo_Fm;
  }
  GraphEntry &k = s->solo_key;
  if (s->solo_slot < 0 || k.h != h || k.u != u || k.Fm != Fm || k.dt != dt || k.nfast != nfast) {
    if (s->solo_slot >= 0) ok(isw_batch_remove(s->solo, s->solo_slot));
    s->solo_slot = -1;
    int slot = -1;
    ok(isw_batch_add(s->solo, s, nullptr, h, u, Fm, nullptr, nullptr, nullptr, 0, dt, nfast, &slot));
    s->solo_slot = slot;
    k = GraphEntry{h, u, Fm, nullptr, dt, nfast, nullptr};
  }
  ok(isw_batch_step(s->solo, st));
}

void layers_step(isw_layers *s, double *h, double *u, double *Fm, double *theta, double dt, int nfast, cudaStream_t st) {
  if (!h || !u) fail(ISW_EINVAL, "layers.step: null h or u");
  if (nfast < 1) fail(ISW_EINVAL, "layers.step: nfast must be >= 1");
  if (!(dt > 0) || !std::isfinite(dt)) fail(ISW_EINVAL, "layers.step: dt must be positive and finite");
  if (s->d.air && !theta) fail(ISW_EINVAL, "layers.step: air layers step with theta (isw_layers_step_air)");
  if (!s->d.air && theta) fail(ISW_EINVAL, "layers.step: theta is for air layers");
  if (s->d.nu4 != 0) s->nu4dt = s->d.nu4 * dt;   // the step's nabla^4 loss, booked as heat by an air exchange
  if (s->d.precision == ISW_MIXED) {
    layers_step_solo(s, h, u, Fm, dt, nfast, st);
    return;
  }
  const LayersDev &D = s->d;
  if (!s->percall && !D.air && !D.wall && !D.ob && !(D.shelf > 0) && !D.sig && !D.tide && !D.cbot && !(D.cd_bot > 0)) {
    cudaStreamCaptureStatus cs0 = cudaStreamCaptureStatusNone;
    ISW_CUDA(cudaStreamIsCapturing(st, &cs0));
    const GraphEntry &k = s->solo_key;
    const bool ready = s->solo && s->solo_slot >= 0 && k.h == h && k.u == u && k.dt == dt && k.nfast == nfast &&
                       (Fm ? k.Fm == Fm : k.Fm == s->solo_Fm);
    // (inside a capture of the caller's the batch cannot be built: the per-call kernels below give the same bits)
    if (cs0 == cudaStreamCaptureStatusNone || ready) {
      layers_step_solo(s, h, u, Fm, dt, nfast, st);
      return;
    }
  }
  auto enqueue = [&](cudaStream_t q) {
    if (s->d.air) enqueue_step_air(s, h, u, Fm, theta, dt, nfast, q);
    else enqueue_step(s, h, u, Fm, dt, nfast, q);
  };
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ISW_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {   // the caller is capturing a graph of its own: just queue the kernels
    enqueue(st);
    return;
  }
  for (auto it = s->graphs.begin(); it != s->graphs.end(); ++it)
    if (it->h == h && it->u == u && it->Fm == Fm && it->theta == theta && it->dt == dt && it->nfast == nfast) {
      s->graphs.splice(s->graphs.begin(), s->graphs, it);
      ISW_CUDA(cudaGraphLaunch(it->exec, st));
      return;
    }
  cudaGraph_t graph = nullptr;
  ISW_CUDA(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue(s->cap);
  } catch (...) {
    cudaStreamEndCapture(s->cap, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  ISW_CUDA(cudaStreamEndCapture(s->cap, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  ISW_CUDA(ie);
  s->graphs.push_front(GraphEntry{h, u, Fm, theta, dt, nfast, exec});
  if (s->graphs.size() > GRAPH_CACHE) {
    cudaGraphExecDestroy(s->graphs.back().exec);
    s->graphs.pop_back();
  }
  ISW_CUDA(cudaGraphLaunch(exec, st));
}

// The between-step exchange (reference layers.py:214-232): thickness, tracer and momentum between layers; for air
// layers (theta given) the momentum mixing's kinetic-energy loss and the step's nabla^4 loss return as heat.
void layers_exchange(isw_layers *s, const double *wx, double *h, double *u, double *Mm, double *psi, double *theta, int seq,
                     cudaStream_t st) {
  if (!wx || !h || !u || !Mm || !psi) fail(ISW_EINVAL, "layers.exchange: null array");
  const LayersDev &M = s->d;
  const int L = M.L, N = M.g.N, E = M.g.E;
  if (L < 2) return;
  const bool heat = M.air && theta;
  const bool v4 = heat && M.nu4 != 0;
  ISW_CUDA(cudaMemcpyAsync(M.hold, h, sizeof(double) * (size_t)L * N, cudaMemcpyDeviceToDevice, st));
  ISW_DISPATCH_L(L, (k_xch_cell<LL><<<blocks_for(N), THREADS, 0, st>>>(M, wx, h, Mm, psi, seq ? 1 : 0)));
  ISW_DISPATCH_L(L, (k_xch_edge<LL><<<blocks_for(E), THREADS, 0, st>>>(M, wx, u, heat ? M.diss : nullptr, v4 ? M.L2 : nullptr,
                                                                       v4 ? s->nu4dt : 0.0, heat ? M.thin_wind : 0.0)));
  if (heat) ISW_DISPATCH_L(L, (k_vmix_heat<LL><<<blocks_for(N), THREADS, 0, st>>>(M, h, theta)));
  ISW_CUDA(cudaGetLastError());
}

void layers_update_gfast(isw_layers *s, const double *h, const double *theta, cudaStream_t st) {
  if (!s->d.air) fail(ISW_EINVAL, "layers.update_gfast: for air layers");
  if (!h || !theta) fail(ISW_EINVAL, "layers.update_gfast: null h or theta");
  ISW_DISPATCH_L(s->d.L, (k_air_gfast<LL><<<blocks_for(s->d.g.N), THREADS, 0, st>>>(s->d, h, theta)));
  ISW_CUDA(cudaGetLastError());
}

int layers_substeps(isw_layers *s, const double *h, double dt, cudaStream_t st) {
  if (!h) fail(ISW_EINVAL, "layers.substeps: null h");
  ISW_CUDA(cudaMemsetAsync(s->nonfinite, 0, sizeof(int), st));
  k_colmax<<<s->colmax_blocks, THREADS, 0, st>>>(s->d, h, s->d.red, s->nonfinite);
  k_max_reduce<<<1, THREADS, 0, st>>>(s->d.red, s->colmax_blocks, s->d.red + s->colmax_blocks);
  ISW_CUDA(cudaGetLastError());
  double c2 = 0;
  int nf = 0;
  ISW_CUDA(cudaMemcpyAsync(&c2, s->d.red + s->colmax_blocks, sizeof(double), cudaMemcpyDeviceToHost, st));
  ISW_CUDA(cudaMemcpyAsync(&nf, s->nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
  ISW_CUDA(cudaStreamSynchronize(st));
  if (nf) fail(ISW_ENOTFINITE, "layers.substeps: non-finite column thickness");
  const double n = std::ceil(dt * std::sqrt(c2) / (0.5 * s->grid->dmin));
  return n > 1 ? (int)n : 1;
}

void layers_lap(isw_layers *s, const double *u, double *out, cudaStream_t st) {
  if (!u || !out) fail(ISW_EINVAL, "layers.lap: null array");
  const LayersDev &M = s->d;
  ISW_DISPATCH_L(M.L, (k_lap_cv<LL><<<blocks_for(M.g.N + M.g.NV), THREADS, 0, st>>>(M, u)));
  ISW_DISPATCH_L(M.L, (k_lap_e<LL><<<blocks_for(M.g.E), THREADS, 0, st>>>(M, out)));
  ISW_CUDA(cudaGetLastError());
}

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

}  // namespace

extern "C" {

int isw_layers_create(isw_grid *g, const isw_layers_params *p, isw_layers **out) {
  return guarded([&] {
    if (!out) fail(ISW_EINVAL, "layers: null output handle");
    *out = layers_create(g, p);
  });
}

int isw_layers_destroy(isw_layers *s) {
  if (s) layers_destroy(s);
  return ISW_OK;
}

int isw_layers_step(isw_layers *s, double *h, double *u, double *Fm, double dt, int nfast, void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.step: null handle");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    layers_step(s, h, u, Fm, nullptr, dt, nfast, (cudaStream_t)stream);
  });
}

int isw_layers_step_air(isw_layers *s, double *h, double *u, double *Fm, double *theta, double dt, int nfast, void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.step: null handle");
    if (!theta) fail(ISW_EINVAL, "layers.step: null theta");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    layers_step(s, h, u, Fm, theta, dt, nfast, (cudaStream_t)stream);
  });
}

int isw_layers_exchange(isw_layers *s, const double *wx, double *h, double *u, double *M, double *psi, double *theta, int seq,
                        void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.exchange: null handle");
    if (s->d.precision != ISW_FP64) fail(ISW_EUNSUPPORTED, "layers.exchange: the FP64 form only");
    if (theta && !s->d.air) fail(ISW_EINVAL, "layers.exchange: theta is for air layers");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    layers_exchange(s, wx, h, u, M, psi, theta, seq, (cudaStream_t)stream);
  });
}

int isw_layers_set_option(isw_layers *s, int option, const double *array, double value) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.set_option: null handle");
    if (s->d.precision != ISW_FP64) fail(ISW_EUNSUPPORTED, "layers.set_option: the FP64 form only");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    LayersDev &d = s->d;
    switch (option) {
      case ISW_OPT_SIG:
        if (array && d.air) fail(ISW_EINVAL, "layers.set_option: per-cell buoyancy is for Boussinesq layers");
        if (array && !d.zm) d.zm = dalloc(s, (size_t)d.L * d.g.N);
        d.sig = array;
        break;
      case ISW_OPT_TIDE: d.tide = array; break;
      case ISW_OPT_CBOT: d.cbot = array; break;
      case ISW_OPT_CD_BOT:
        if (!(value >= 0)) fail(ISW_EINVAL, "layers.set_option: cd_bot must be >= 0");
        d.cd_bot = value;
        break;
      default: fail(ISW_EINVAL, "layers.set_option: unknown option");
    }
    for (auto &e : s->graphs) cudaGraphExecDestroy(e.exec);   // the step graphs hold the old descriptor
    s->graphs.clear();
    s->version++;
  });
}

int isw_layers_update_gfast(isw_layers *s, const double *h, const double *theta, void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.update_gfast: null handle");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    layers_update_gfast(s, h, theta, (cudaStream_t)stream);
  });
}

int isw_layers_substeps(isw_layers *s, const double *h, double dt, int *out, void *stream) {
  return guarded([&] {
    if (!s || !out) fail(ISW_EINVAL, "layers.substeps: null handle or output");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    *out = layers_substeps(s, h, dt, (cudaStream_t)stream);
  });
}

int isw_layers_vmix_heat(isw_layers *s, const double *h, const double *diss, double *theta, double grav, double cp,
                         double kappa, double p0, void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.vmix_heat: null handle");
    if (!h || !diss || !theta) fail(ISW_EINVAL, "layers.vmix_heat: null array");
    if (!(p0 > 0) || !(kappa > -1) || !std::isfinite(grav) || !std::isfinite(cp))
      fail(ISW_EINVAL, "layers.vmix_heat: p0 must be positive, kappa > -1, grav and cp finite");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    const GridDev &g = s->d.g;
    cudaStream_t st = (cudaStream_t)stream;
    ISW_DISPATCH_L(s->d.L, (k_heat<LL><<<blocks_for(g.N), THREADS, 0, st>>>(g, h, diss, grav, cp, kappa, p0, theta)));
    ISW_CUDA(cudaGetLastError());
  });
}

int isw_layers_mask(isw_layers *s, double *a, int rows, void *stream) {
  return guarded([&] {
    if (!s || !a) fail(ISW_EINVAL, "layers.mask: null handle or array");
    if (rows < 1 || rows > LMAX) fail(ISW_EINVAL, "layers.mask: rows outside 1..8");
    if (!s->d.wall) return;                     // no walls: nothing to zero
    ISW_CUDA(cudaSetDevice(s->grid->device));
    const int E = s->d.g.E;
    k_wall_mask<<<blocks_for(E), THREADS, 0, (cudaStream_t)stream>>>(s->d.wall, E, rows, a);
    ISW_CUDA(cudaGetLastError());
  });
}

int isw_layers_set_bottom(isw_layers *s, const double *b, void *stream) {
  return guarded([&] {
    if (!s || !b) fail(ISW_EINVAL, "layers.set_bottom: null handle or array");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    ISW_CUDA(cudaMemcpyAsync(const_cast<double *>(s->d.b), b, sizeof(double) * (size_t)s->d.g.N, cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
  });
}

int isw_layers_status(isw_layers *s, void *stream, int reset) {
  if (!s) {
    set_last_error("layers.status: null handle");
    return ISW_EINVAL;
  }
  if (!s->solo) return ISW_OK;                  // only the batched one-stack path keeps a status word
  return isw_batch_status(s->solo, stream, reset);
}

int isw_layers_lap(isw_layers *s, const double *u, double *out, void *stream) {
  return guarded([&] {
    if (!s) fail(ISW_EINVAL, "layers.lap: null handle");
    ISW_CUDA(cudaSetDevice(s->grid->device));
    layers_lap(s, u, out, (cudaStream_t)stream);
  });
}

}  // extern "C"
