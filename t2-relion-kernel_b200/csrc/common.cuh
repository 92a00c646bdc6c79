// common.cuh -- shared device helpers of the coarse-pass diff2 library.
//
// Reference correspondence (Edgarrrrrr/T2-RELION-kernel):
//   rotate_pixel / project_pixel : AccProjectorKernel::project3Dmodel
//                                  (src/acc_projectorkernel_impl.h:178-252)
//   trilinear_linear             : no_tex3D (src/cuda_device_utils.cuh:73-108)
//   pixel_coor                   : pixel_index2coor (src/diff2.cuh:182-188)
//   translate_pixel              : translatePixel (src/cuda_device_utils.cuh:110-129)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include <nvtx3/nvToolsExt.h>

#include "../../include/b200d2.h"

namespace b200d2 {

#define B200D2_CUDA_TRY(expr)                                   \
  do {                                                          \
    cudaError_t e_ = (expr);                                    \
    if (e_ != cudaSuccess) return b200d2::status_from_cuda(e_); \
  } while (0)

// Process-wide count of kernel launches made by this library.
void count_launch(unsigned n = 1);

// Counter advanced whenever a projector is created or destroyed: state keyed
// on a projector view (whose texture handles a later projector may reuse) is
// valid only while it is unchanged.
unsigned long long projector_epoch();

// Blocks of the projection cache's check of the Euler matrices: block b
// writes its verdict to word b, and the projection stage ORs the words.
constexpr int kEulCheckBlocks = 64;

// NVTX range over a host scope (a batch call, a pipeline stage, a served
// request), so that a timeline profiler labels the library's launches; without
// a profiler attached the push and pop cost a few nanoseconds.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Opts `kernel` in to `bytes` of dynamic shared memory on the current device,
// once per device (the attribute belongs to each device's context); `done`
// holds one bit per device ordinal (mod 64).
template <typename K>
inline cudaError_t smem_opt_in(K* kernel, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load() & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit);
  return e;
}

inline int status_from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return B200D2_OK;
  if (e == cudaErrorMemoryAllocation) return B200D2_ERR_OOM;
  return B200D2_ERR_CUDA;
}

// Precisions served by the tensor-core pipeline.
inline bool is_tc_precision(int p) {
  return p == B200D2_PREC_TF32 || p == B200D2_PREC_TF32X3 || p == B200D2_PREC_BF16X3 ||
         p == B200D2_PREC_FP16 || p == B200D2_PREC_FP16X3;
}

// Sample positions are formed with explicit, ordered fused multiply-adds so
// that every kernel of this library (and the CPU oracle, which uses the same
// order) sees bit-identical coordinates:
//   xp = fma(e0, x, e1*y) * pf        r2 = (int) fma(zp, zp, fma(xp, xp, yp*yp))
struct Rotated {
  float xp, yp, zp;
  int r2;
};

__device__ __forceinline__ Rotated rotate_pixel(float fx, float fy, float e0,
                                                float e1, float e3, float e4,
                                                float e6, float e7, float pf) {
  Rotated r;
  r.xp = __fmul_rn(__fmaf_rn(e0, fx, __fmul_rn(e1, fy)), pf);
  r.yp = __fmul_rn(__fmaf_rn(e3, fx, __fmul_rn(e4, fy)), pf);
  r.zp = __fmul_rn(__fmaf_rn(e6, fx, __fmul_rn(e7, fy)), pf);
  r.r2 = (int)__fmaf_rn(r.zp, r.zp, __fmaf_rn(r.xp, r.xp, __fmul_rn(r.yp, r.yp)));
  return r;
}

__device__ __forceinline__ float lerp_f(float a, float b, float t) {
  return __fmaf_rn(__fsub_rn(b, a), t, a);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// Software trilinear on a linear [mdlZ][mdlY][mdlX] array with exact FP32
// weights: the reference's no_tex3D arithmetic (indices clamped to the array,
// which equals the reference wherever its reads are in bounds).
__device__ __forceinline__ float trilinear_linear(const float* __restrict__ mdl,
                                                  float xp, float yp, float zp,
                                                  int mdlX, int mdlY, int mdlZ,
                                                  int mdlInitY, int mdlInitZ) {
  float fx0 = floorf(xp), fy0 = floorf(yp), fz0 = floorf(zp);
  float fx = __fsub_rn(xp, fx0), fy = __fsub_rn(yp, fy0), fz = __fsub_rn(zp, fz0);
  int x0 = (int)fx0, y0 = (int)fy0 - mdlInitY, z0 = (int)fz0 - mdlInitZ;
  int x1 = clampi(x0 + 1, 0, mdlX - 1), y1 = clampi(y0 + 1, 0, mdlY - 1),
      z1 = clampi(z0 + 1, 0, mdlZ - 1);
  x0 = clampi(x0, 0, mdlX - 1);
  y0 = clampi(y0, 0, mdlY - 1);
  z0 = clampi(z0, 0, mdlZ - 1);
  const size_t sxy = (size_t)mdlX * mdlY;
  const float* p00 = mdl + z0 * sxy + (size_t)y0 * mdlX;
  const float* p01 = mdl + z0 * sxy + (size_t)y1 * mdlX;
  const float* p10 = mdl + z1 * sxy + (size_t)y0 * mdlX;
  const float* p11 = mdl + z1 * sxy + (size_t)y1 * mdlX;
  float dx00 = lerp_f(__ldg(p00 + x0), __ldg(p00 + x1), fx);
  float dx01 = lerp_f(__ldg(p10 + x0), __ldg(p10 + x1), fx);
  float dx10 = lerp_f(__ldg(p01 + x0), __ldg(p01 + x1), fx);
  float dx11 = lerp_f(__ldg(p11 + x0), __ldg(p11 + x1), fx);
  float dxy0 = lerp_f(dx00, dx10, fy);
  float dxy1 = lerp_f(dx01, dx11, fy);
  return lerp_f(dxy0, dxy1, fz);
}

// project3Dmodel for a 2D image pixel into the 3D reference.  `e` holds the
// six used Euler entries (e0, e1, e3, e4, e6, e7).
__device__ __forceinline__ float2 project_pixel(const b200d2_view& v, float fx,
                                                float fy, const float* e) {
  Rotated r = rotate_pixel(fx, fy, e[0], e[1], e[2], e[3], e[4], e[5],
                           v.padding_factor);
  float2 out = make_float2(0.f, 0.f);
  if (r.r2 <= v.maxR2_padded) {
    float xp = r.xp, yp = r.yp, zp = r.zp, sgn = 1.f;
    if (xp < 0.f) {  // Hermitian conjugate pair
      xp = -xp;
      yp = -yp;
      zp = -zp;
      sgn = -1.f;
    }
    if (v.interp == B200D2_INTERP_TEXTURE) {
      yp = __fsub_rn(yp, (float)v.mdlInitY);
      zp = __fsub_rn(zp, (float)v.mdlInitZ);
      float u = __fadd_rn(xp, 0.5f), w1 = __fadd_rn(yp, 0.5f),
            w2 = __fadd_rn(zp, 0.5f);
      if (v.tex_c) {  // one fetch of both channels
        const float2 t = tex3D<float2>((cudaTextureObject_t)v.tex_c, u, w1, w2);
        out.x = t.x;
        out.y = sgn * t.y;
      } else {
        out.x = tex3D<float>((cudaTextureObject_t)v.tex_re, u, w1, w2);
        out.y = sgn * tex3D<float>((cudaTextureObject_t)v.tex_im, u, w1, w2);
      }
    } else {
      const int mdlY = v.mdlXY / v.mdlX;
      out.x = trilinear_linear(v.lin_re, xp, yp, zp, v.mdlX, mdlY, v.mdlZ,
                               v.mdlInitY, v.mdlInitZ);
      out.y = sgn * trilinear_linear(v.lin_im, xp, yp, zp, v.mdlX, mdlY,
                                     v.mdlZ, v.mdlInitY, v.mdlInitZ);
    }
  }
  return out;
}

// pixel_index2coor
__device__ __forceinline__ void pixel_coor(int idx, int imgX, int imgY,
                                           int maxR, int& x, int& y) {
  x = idx % imgX;
  y = idx / imgX;
  if (y > maxR) y -= imgY;
}

// Superset of the pixels that any orientation can place inside the projector
// radius: int(fp32 |pf R (x,y,0)|^2) <= maxR2_padded needs the float value to
// be below maxR2_padded + 1, and the float value differs from the exact
// pf^2 (x^2 + y^2) by far less than one unit for every supported size.
__host__ __device__ __forceinline__ bool pixel_maybe_inside(int x, int y,
                                                            float pf,
                                                            int maxR2_padded) {
  double r2 = (double)(x * x + y * y) * (double)pf * (double)pf;
  return r2 < (double)maxR2_padded + 2.0;
}

// Merged batches: several requests on one reference in one stream-ordered
// pipeline run, each request's particles against its own orientation columns
// (tc_pipeline.cu; used by the serving loop).
struct MergedRequest {
  int P, O, T;  // particles, orientations, translations
  int col0;     // first column of its orientations in the merged set: a multiple of 256, increasing
  const float* h_tx;  // host [T] phase slopes
  const float* h_ty;
};
struct MergedDev {
  const float* re;  // device [P][N_img]
  const float* im;
  const float* corr;
  float* out;  // device [P][O][T]
};
struct MergedBatch;
// Host-side tables of the batch (no CUDA calls); null with *status set when invalid.
MergedBatch* merged_create(const b200d2_view& v, int N_img, int precision, const MergedRequest* r, int n,
                           int O_cols, int* status);
// Device bytes (workspace and tables) and page-locked staging bytes (tables) of a run.
size_t merged_device_bytes(const MergedBatch* m);
size_t merged_host_bytes(const MergedBatch* m);
// Copy the tables from `hstage` (page-locked, 256-byte aligned, merged_host_bytes)
// into `dmem` (256-byte aligned, merged_device_bytes) and launch every stage on s.
// d_eulers: [O_cols][9] device; d_min / d_argmin: device [sum of P] in request order.
int merged_enqueue(MergedBatch* m, const float* d_eulers, const MergedDev* d, double* d_min, long long* d_argmin,
                   void* dmem, void* hstage, cudaStream_t s);
void merged_destroy(MergedBatch* m);

// Load every kernel the tensor-core pipeline of `precision` can launch
// (instead of at its first launch, which can wait for running work).
int tc_preload(int precision);

}  // namespace b200d2
