// weights.cu -- coarse-pass weights: per-particle exp(-(diff2 - min)) in FP64,
// their deterministic per-particle sums and normalisation.
//
// Reference: the step after the coarse pass in RELION's E-step, whose driver
// kernel_weights_exponent_coarse is a commented stub in the reference harness
// (src/utilities.h:405-443: per sample pdf_orientation * pdf_offset *
// exp(-(diff2 - min_diff2)) over nr_coarse_orient x nr_coarse_trans samples;
// a zero prior gives a zero weight here).
//
// Layout: diff2[p][o][t] (the coarse output), n = O*T samples per particle.
// Each particle's block is cut into fixed chunks of kChunk samples; a CTA sums
// one chunk in a fixed order and the last CTA of a particle (completion
// counter) adds the chunk sums in chunk order, so sums are bit-reproducible.
// Every kernel streams diff2 once from HBM: the bound is HBM bandwidth.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace b200d2 {

constexpr int kWThreads = 256;
constexpr long long kChunk = 32768;

int minloc(const float* d, long long n, int P, double* mn, long long* arg, cudaStream_t s);

__device__ __forceinline__ double weight_at(const float* __restrict__ row, long long i, int T, double mn,
                                            const double* __restrict__ pdf_o,
                                            const double* __restrict__ pdf_t) {
  double w = exp(-((double)row[i] - mn));
  if (pdf_o) w *= pdf_o[i / T];
  if (pdf_t) w *= pdf_t[i % T];
  return w;
}

// Sum over the CTA in a fixed order (shuffle tree, then warps in order).
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s_part[kWThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kWThreads / 32; ++w) t += s_part[w];
  return t;
}

__global__ void __launch_bounds__(kWThreads) weights_sum_kernel(const float* __restrict__ d2, long long n, int T,
                                                                const double* __restrict__ mn,
                                                                const double* __restrict__ pdf_o,
                                                                const double* __restrict__ pdf_t, double* partial,
                                                                unsigned* count, int nchunk, double* sum) {
  const int p = blockIdx.y, c = blockIdx.x;
  const float* row = d2 + (long long)p * n;
  const double m = mn[p];
  const long long lo = (long long)c * kChunk, hi = min(n, lo + kChunk);
  double acc = 0.0;
  for (long long i = lo + threadIdx.x; i < hi; i += kWThreads) acc += weight_at(row, i, T, m, pdf_o, pdf_t);
  acc = block_sum(acc);
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    partial[(long long)p * nchunk + c] = acc;
    __threadfence();
    s_last = atomicAdd(&count[p], 1u) == (unsigned)(nchunk - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    const volatile double* pp = partial + (long long)p * nchunk;
    double s = 0.0;
    for (int k = 0; k < nchunk; ++k) s += pp[k];
    sum[p] = s;
    count[p] = 0;  // ready for the next call
  }
}

__global__ void __launch_bounds__(kWThreads) weights_write_kernel(const float* __restrict__ d2, long long n, int T,
                                                                  const double* __restrict__ mn,
                                                                  const double* __restrict__ pdf_o,
                                                                  const double* __restrict__ pdf_t,
                                                                  const double* __restrict__ sum, int normalize,
                                                                  double* __restrict__ w) {
  const int p = blockIdx.y;
  const float* row = d2 + (long long)p * n;
  double* out = w + (long long)p * n;
  const double m = mn[p], s = sum[p];
  const long long lo = (long long)blockIdx.x * kChunk, hi = min(n, lo + kChunk);
  for (long long i = lo + threadIdx.x; i < hi; i += kWThreads) {
    const double v = weight_at(row, i, T, m, pdf_o, pdf_t);
    out[i] = normalize ? v / s : v;
  }
}

static inline size_t wal(size_t v) { return (v + 255) / 256 * 256; }

static int nchunks(long long n) { return (int)((n + kChunk - 1) / kChunk); }

}  // namespace b200d2

extern "C" size_t b200d2_coarse_weights_workspace(int P, long long n) {
  using namespace b200d2;
  if (P <= 0 || n <= 0) return 0;
  return wal(sizeof(double) * P) + wal(sizeof(double) * (size_t)P * nchunks(n)) + wal(sizeof(unsigned) * P);
}

extern "C" int b200d2_coarse_weights(const float* d_diff2, int P, int O, int T, const double* d_min,
                                     const double* d_pdf_orient, const double* d_pdf_offset, int normalize,
                                     double* d_weights, double* d_sum, void* d_workspace, size_t workspace_bytes,
                                     void* stream) {
  using namespace b200d2;
  if (P < 0 || O < 0 || T < 0) return B200D2_ERR_INVALID;
  const long long n = (long long)O * T;
  if (P == 0 || n == 0) return B200D2_OK;
  if (!d_diff2 || !d_sum || (!d_weights && normalize)) return B200D2_ERR_INVALID;
  if (P > 65535 || nchunks(n) > 0x7fffffff) return B200D2_ERR_UNSUPPORTED;
  const size_t need = b200d2_coarse_weights_workspace(P, n);
  if (!d_workspace || workspace_bytes < need) return B200D2_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  uint8_t* ws = static_cast<uint8_t*>(d_workspace);
  double* mn = reinterpret_cast<double*>(ws);
  double* partial = reinterpret_cast<double*>(ws + wal(sizeof(double) * P));
  unsigned* count = reinterpret_cast<unsigned*>(ws + wal(sizeof(double) * P) +
                                                wal(sizeof(double) * (size_t)P * nchunks(n)));
  if (d_min) {
    B200D2_CUDA_TRY(cudaMemcpyAsync(mn, d_min, sizeof(double) * P, cudaMemcpyDeviceToDevice, s));
  } else {
    const int st = minloc(d_diff2, n, P, mn, nullptr, s);
    if (st != B200D2_OK) return st;
  }
  B200D2_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(unsigned) * P, s));
  const dim3 grid(nchunks(n), P);
  weights_sum_kernel<<<grid, kWThreads, 0, s>>>(d_diff2, n, T, mn, d_pdf_orient, d_pdf_offset, partial, count,
                                                nchunks(n), d_sum);
  count_launch();
  B200D2_CUDA_TRY(cudaGetLastError());
  if (d_weights) {
    weights_write_kernel<<<grid, kWThreads, 0, s>>>(d_diff2, n, T, mn, d_pdf_orient, d_pdf_offset, d_sum,
                                                    normalize, d_weights);
    count_launch();
    B200D2_CUDA_TRY(cudaGetLastError());
  }
  return B200D2_OK;
}
