// maskpack.cu -- significance mask packed to bits for the host.
//
// b200d2_significance writes RELION's pass-0 mask as one byte per sample, as
// the reference's cuda_kernel_array_over_threshold does
// (src/cuda_device_utils.cuh:254-266).  RELION reads that mask back to the
// host to build the fine pass's job lists; packed to one bit per sample the
// copy is eight times smaller.  Word j of particle p holds samples
// 32 j .. 32 j + 31 of the particle, sample 32 j + i in bit i (the order of
// numpy's packbits(..., bitorder="little") read as little-endian 32-bit
// words); bits past n are zero.  One thread per word: a warp reads 1 KiB of
// consecutive mask bytes and writes 128 consecutive bytes of words.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace b200d2 {

// bits i of the result: byte i of v is non-zero (4 bytes)
__device__ __forceinline__ uint32_t nonzero_bytes(uint32_t v) {
  return (uint32_t)((v & 0x000000ffu) != 0) | ((uint32_t)((v & 0x0000ff00u) != 0) << 1) |
         ((uint32_t)((v & 0x00ff0000u) != 0) << 2) | ((uint32_t)((v & 0xff000000u) != 0) << 3);
}

// VEC: every word's 32 bytes are 16-byte aligned and inside the row (n a
// multiple of 16, 16-byte aligned base); otherwise bytes are read one by one.
template <bool VEC>
__global__ void __launch_bounds__(256) pack_mask_kernel(const uint8_t* __restrict__ mask, long long n,
                                                        long long words_per_p, long long total,
                                                        uint32_t* __restrict__ bits) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const long long p = w / words_per_p, j = w - p * words_per_p;
    const long long i0 = 32 * j;
    const uint8_t* src = mask + p * n + i0;
    uint32_t out = 0;
    if (VEC && i0 + 32 <= n) {
      const uint4 a = reinterpret_cast<const uint4*>(src)[0];
      const uint4 b = reinterpret_cast<const uint4*>(src)[1];
      const uint32_t q[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int k = 0; k < 8; ++k) out |= nonzero_bytes(q[k]) << (4 * k);
    } else {
      const int cnt = (int)min(32LL, n - i0);
      for (int k = 0; k < cnt; ++k) out |= (uint32_t)(src[k] != 0) << k;
    }
    bits[w] = out;
  }
}

int pack_mask(const uint8_t* mask, int P, long long n, uint32_t* bits, cudaStream_t s) {
  if (P == 0 || n == 0) return B200D2_OK;
  const long long wpp = (n + 31) / 32, total = (long long)P * wpp;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  const bool vec = n % 16 == 0 && (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
  if (vec)
    pack_mask_kernel<true><<<blocks, 256, 0, s>>>(mask, n, wpp, total, bits);
  else
    pack_mask_kernel<false><<<blocks, 256, 0, s>>>(mask, n, wpp, total, bits);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

}  // namespace b200d2

extern "C" int b200d2_pack_mask(const unsigned char* d_mask, int P, long long n, unsigned int* d_bits,
                                void* stream) {
  if (P < 0 || n < 0) return B200D2_ERR_INVALID;
  if ((P > 0 && n > 0) && (!d_mask || !d_bits)) return B200D2_ERR_INVALID;
  return b200d2::pack_mask(d_mask, P, n, d_bits, (cudaStream_t)stream);
}
