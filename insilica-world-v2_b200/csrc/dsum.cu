// Deterministic sums (reference src/insilica/gpu.py:111-126 and kernels/trisk.cu:61-81): a fixed-order tree, so totals
// are bit-identical run to run and equal to the reference's. Each block reduces 2048 consecutive values: thread t adds
// x[base + t + 256 k] for k = 0..7 in order, then the 256 partial sums halve pairwise, s[t] += s[t + h] for
// h = 128, 64, 32 through shared memory and h = 16 .. 1 by warp shuffles (the same additions in the same order).
// Passes repeat over the block sums until one value remains; all passes are queued at once (the sizes are known).
#include <mutex>

#include "common.cuh"

namespace isw {
namespace {

constexpr int SUM_THREADS = 256, SUM_CHUNK = 8;

__global__ void __launch_bounds__(SUM_THREADS) k_block_sum(long long n, const double *__restrict__ x, const double *__restrict__ y,
                                                           double *__restrict__ out) {
  __shared__ double s[SUM_THREADS];
  const long long base = (long long)blockIdx.x * SUM_THREADS * SUM_CHUNK;
  double acc = 0;
#pragma unroll
  for (int k = 0; k < SUM_CHUNK; k++) {
    const long long i = base + threadIdx.x + (long long)k * SUM_THREADS;
    if (i < n) acc += y ? x[i] * y[i] : x[i];
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < 128) s[threadIdx.x] += s[threadIdx.x + 128];
  __syncthreads();
  if (threadIdx.x < 64) s[threadIdx.x] += s[threadIdx.x + 64];
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = s[threadIdx.x] + s[threadIdx.x + 32];
#pragma unroll
    for (int h = 16; h > 0; h >>= 1) v += __shfl_down_sync(0xffffffffu, v, h);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
  }
}

}  // namespace

long long dsum_blocks(long long n) { return (n + SUM_THREADS * SUM_CHUNK - 1) / (SUM_THREADS * SUM_CHUNK); }

// Scratch doubles the passes need for n values (pass outputs laid end to end).
long long dsum_scratch(long long n) {
  long long tot = 0, m = n;
  do {
    m = dsum_blocks(m);
    tot += m;
  } while (m > 1);
  return tot;
}

// Queue every pass on st; the sum ends in *result (device). scratch holds dsum_scratch(n) doubles.
void dsum_enqueue(const double *x, const double *y, long long n, double *scratch, double *result, cudaStream_t st) {
  long long m = n;
  const double *in = x;
  const double *iy = y;
  double *out = scratch;
  for (;;) {
    const long long b = dsum_blocks(m);
    double *dst = b == 1 ? result : out;
    k_block_sum<<<(unsigned)b, SUM_THREADS, 0, st>>>(m, in, iy, dst);
    if (b == 1) break;
    in = dst;
    iy = nullptr;
    out = dst + b;
    m = b;
  }
  ISW_CUDA(cudaGetLastError());
}

}  // namespace isw

using namespace isw;

extern "C" int isw_dsum(const double *x, const double *y, long long n, double *out, void *stream) {
  try {
    if (!x || !out) fail(ISW_EINVAL, "dsum: null argument");
    if (n < 1) fail(ISW_EINVAL, "dsum: n must be >= 1");
    cudaStream_t st = (cudaStream_t)stream;
    const long long need = dsum_scratch(n) + 1;
    double *buf = nullptr;
    ISW_CUDA(cudaMallocAsync((void **)&buf, sizeof(double) * need, st));
    try {
      dsum_enqueue(x, y, n, buf + 1, buf, st);
      ISW_CUDA(cudaMemcpyAsync(out, buf, sizeof(double), cudaMemcpyDeviceToHost, st));
    } catch (...) {
      cudaFreeAsync(buf, st);
      throw;
    }
    ISW_CUDA(cudaFreeAsync(buf, st));
    ISW_CUDA(cudaStreamSynchronize(st));
    return ISW_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  }
}

// ---- The deterministic sum without any allocation ----
//
// For callers that cannot allocate device memory when they sum: hosts that reserve all device memory up front and
// forbid later cudaMalloc calls (an embedding framework with its own memory pool, a real-time loop that must not stall
// on the allocator), and plugins whose host owns the device heap. The passes' partial sums live in one file-scope
// device array of a fixed size, sized for sums of up to 134,217,728 values (2^27). Every GPU that loads this library
// holds the array until the process exits.
//
// In host code `g_dsum_static` is only a host-side stand-in for the device array, never a device address: the address
// is looked up with cudaGetSymbolAddress once per device, on the first call made with that device current (so that first
// call should come before any stream capture). Every call shares the array and finds in it what the last call left:
// each pass writes every partial sum it later reads, so nothing needs clearing, but calls whose work overlaps on the
// GPU (different streams, or different host threads on one device) race on the array and must be serialised.
namespace isw {
namespace {

constexpr long long DSUM_STATIC_MAX_N = 1LL << 27;                // 134,217,728 values
constexpr long long DSUM_STATIC_SCRATCH = 65536 + 32 + 8;          // dsum_scratch(DSUM_STATIC_MAX_N), with room to spare
constexpr int DSUM_STATIC_DEVICES = 64;

static __device__ __align__(256) double g_dsum_static[DSUM_STATIC_SCRATCH];

std::mutex g_dsum_static_mu;
double *g_dsum_static_addr[DSUM_STATIC_DEVICES] = {};

double *dsum_static_scratch() {
  int dev = -1;
  ISW_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= DSUM_STATIC_DEVICES) fail(ISW_EINVAL, "dsum_static: device index beyond 63");
  std::lock_guard<std::mutex> lock(g_dsum_static_mu);
  if (!g_dsum_static_addr[dev]) {
    double *p = nullptr;
    ISW_CUDA(cudaGetSymbolAddress((void **)&p, g_dsum_static));
    if (!p) fail(ISW_ECUDA, "dsum_static: no device address for the scratch array");
    g_dsum_static_addr[dev] = p;
  }
  return g_dsum_static_addr[dev];
}

}  // namespace
}  // namespace isw

extern "C" int isw_dsum_static(const double *x, const double *y, long long n, double *out, void *stream) {
  try {
    if (!x || !out) fail(ISW_EINVAL, "dsum_static: null argument");
    if (n < 1) fail(ISW_EINVAL, "dsum_static: n must be >= 1");
    if (n > DSUM_STATIC_MAX_N) fail(ISW_EINVAL, "dsum_static: n exceeds the 134217728 values its fixed scratch holds; use isw_dsum");
    if (dsum_scratch(n) > DSUM_STATIC_SCRATCH) fail(ISW_EINVAL, "dsum_static: scratch too small for n");
    dsum_enqueue(x, y, n, dsum_static_scratch(), out, (cudaStream_t)stream);
    return ISW_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  }
}
