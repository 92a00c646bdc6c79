// tex_probe.cu -- samples a 3D float texture object at given coordinates.
//
// TEST INFRASTRUCTURE ONLY: lets the tests compare the texture unit's linear
// filtering with the oracle's CPU emulation sample by sample (an in-bounds
// check of the hardware interpolation's rounding).  Not part of the product.
#include <cuda_runtime.h>

__global__ void texprobe_kernel(cudaTextureObject_t tex, const float* __restrict__ uvw, int n,
                                float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex3D<float>(tex, uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2]);
}

extern "C" int texprobe_sample(unsigned long long tex, const float* d_uvw, int n, float* d_out,
                               void* stream) {
  if (n <= 0) return 0;
  texprobe_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>((cudaTextureObject_t)tex, d_uvw,
                                                                      n, d_out);
  return (int)cudaGetLastError();
}
