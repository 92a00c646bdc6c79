// minloc.cu -- per-particle minimum diff2 and its (o, t) index.
//
// No counterpart in the reference harness (RELION computes the minimum on the
// host after the coarse pass).  One CTA per particle reduces n floats: each
// thread keeps the smallest (value, index) pair it sees, then a warp-shuffle
// and a shared-memory step combine them; ties resolve to the lowest index, so
// the result is deterministic.
#include <cuda_runtime.h>

#include "common.cuh"

namespace b200d2 {

__device__ __forceinline__ void better(float& v, long long& i, float v2, long long i2) {
  if (v2 < v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

__global__ void __launch_bounds__(512) minloc_kernel(const float* __restrict__ d, long long n,
                                                     double* __restrict__ out_min,
                                                     long long* __restrict__ out_arg) {
  const float* row = d + (long long)blockIdx.x * n;
  float v = __int_as_float(0x7f800000);  // +inf
  long long idx = 0x7fffffffffffffffLL;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = row[i];
    if (x < v) {  // strictly smaller keeps the first (lowest) index per thread
      v = x;
      idx = i;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float v2 = __shfl_xor_sync(0xffffffffu, v, o);
    long long i2 = __shfl_xor_sync(0xffffffffu, idx, o);
    better(v, idx, v2, i2);
  }
  __shared__ float sv[16];
  __shared__ long long si[16];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sv[warp] = v;
    si[warp] = idx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) better(v, idx, sv[w], si[w]);
    if (out_min) out_min[blockIdx.x] = (double)v;
    if (out_arg) out_arg[blockIdx.x] = idx;
  }
}

int minloc(const float* d, long long n, int P, double* mn, long long* arg, cudaStream_t s) {
  if (P <= 0 || n <= 0) return B200D2_OK;
  minloc_kernel<<<P, 512, 0, s>>>(d, n, mn, arg);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

}  // namespace b200d2

extern "C" int b200d2_minloc(const float* d_diff2, long long n, int P, double* d_min,
                             long long* d_argmin, void* stream) {
  if (!d_diff2 || n < 0 || P < 0) return B200D2_ERR_INVALID;
  if (P > 0x7fffffff) return B200D2_ERR_INVALID;
  return b200d2::minloc(d_diff2, n, P, d_min, d_argmin, (cudaStream_t)stream);
}
