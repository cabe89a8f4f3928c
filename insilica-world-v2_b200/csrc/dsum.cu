// Deterministic sums (reference src/insilica/gpu.py:111-126 and kernels/trisk.cu:61-81): a fixed-order tree, so totals
// are bit-identical run to run and equal to the reference's. Each block reduces 2048 consecutive values: thread t adds
// x[base + t + 256 k] for k = 0..7 in order, then the 256 partial sums halve pairwise, s[t] += s[t + h] for
// h = 128, 64, 32 through shared memory and h = 16 .. 1 by warp shuffles (the same additions in the same order).
// Passes repeat over the block sums until one value remains; all passes are queued at once (the sizes are known).
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
