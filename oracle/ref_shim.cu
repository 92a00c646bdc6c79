// ref_shim.cu -- C entry points around the reference project's own CUDA code.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit is compiled by
// oracle/Makefile against the reference sources where they lie
// (Edgarrrrrr/T2-RELION-kernel, src/*.cuh / src/*.h) into oracle/_ref/.  It
// contains no reference code itself: it includes the reference headers and
// exposes their entry points with plain C signatures so that the parity tests
// can run the reference kernels on the same device buffers as this
// repository's kernels.  Nothing in the product links or loads it.
//
// Wrapped entry points (reference file:line):
//   AccProjector::setMdlDim / initMdl         src/acc_projector_impl.h:10-216
//   AccProjectorKernel::makeKernel            src/acc_projectorkernel_impl.h:410-433
//   runDiff2KernelCoarse                      src/acc_helper_functions_impl.h:15-499
//   runDiff2KernelCoarseDouble                src/acc_helper_functions_impl.h:503-854
//   CoarseMatrixKernel*::run (5 variants)     src/coarse_splitImg_*.cuh
//   cuda_kernel_diff2_fine (no host wrapper)  src/diff2.cuh:540-682
//   cuda_kernel_diff2_CC_fine (no host wrapper) src/diff2.cuh:811-960
//   runDiff2KernelCoarse with do_CC           src/acc_helper_functions_impl.h:441-498
//   cuda_kernel_find_threshold_idx_in_cumulative,
//   cuda_kernel_array_over_threshold          src/cuda_device_utils.cuh:238-266
// The reference's texture projector is used.  Its PROJECTOR_NO_TEXTURES
// configuration does not compile (src/diff2.cuh:16 includes
// src/orientation_matrix_handler.cuh, which calls tex3D unconditionally at
// :144-145), so that path cannot be run as a checker.
#include <cuda_runtime.h>

// standard headers the reference headers expect to be included first
#include <algorithm>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "acc_helper_functions_impl.h"
#include "acc_projector.h"
#include "acc_projector_impl.h"
#include "acc_projectorkernel_impl.h"
#include "coarse_kernel.cuh"
#include "diff2.cuh"

namespace {
struct RefProjector {
  AccProjector proj;
  int mdlX, mdlY, mdlZ;
};

AccProjectorKernel make_view(RefProjector* p, int imgX, int imgY, int imgZ,
                             int imgMaxR) {
  return AccProjectorKernel::makeKernel(p->proj, imgX, imgY, imgZ, imgMaxR);
}
}  // namespace

extern "C" {

int refshim_abi_version(void) { return 6; }

void* refshim_projector_create(int mdlX, int mdlY, int mdlZ, int initY,
                               int initZ, int maxR, float pf, const float* re,
                               const float* im) {
  RefProjector* p = new RefProjector();
  p->mdlX = mdlX;
  p->mdlY = mdlY;
  p->mdlZ = mdlZ;
  p->proj.setMdlDim(mdlX, mdlY, mdlZ, initY, initZ, maxR, pf);
  p->proj.initMdl(const_cast<float*>(re), const_cast<float*>(im));
  if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
  return p;
}

void refshim_projector_destroy(void* h) {
  delete reinterpret_cast<RefProjector*>(h);
}

int refshim_diff2_coarse(void* h, int imgX, int imgY, int imgZ, int imgMaxR,
                         float* d_eulers, float* d_tx, float* d_ty,
                         float* d_corr, float* d_re, float* d_im,
                         float* d_diff2s, long O, long T, long N_img,
                         void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  runDiff2KernelCoarse(k, d_tx, d_ty, nullptr, d_corr, d_re, d_im, d_eulers,
                       d_diff2s, 1.f, (unsigned long)O, (unsigned long)T,
                       (unsigned long)N_img, (cudaStream_t)stream, false,
                       false);
  return (int)cudaGetLastError();
}

// runDiff2KernelCoarse with do_CC (cuda_kernel_diff2_CC_coarse, src/diff2.cuh:691-809)
int refshim_diff2_coarse_cc(void* h, int imgX, int imgY, int imgZ, int imgMaxR,
                            float* d_eulers, float* d_tx, float* d_ty,
                            float* d_corr, float* d_re, float* d_im,
                            float* d_diff2s, long O, long T, long N_img,
                            void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  runDiff2KernelCoarse(k, d_tx, d_ty, nullptr, d_corr, d_re, d_im, d_eulers,
                       d_diff2s, 1.f, (unsigned long)O, (unsigned long)T,
                       (unsigned long)N_img, (cudaStream_t)stream, true,
                       false);
  return (int)cudaGetLastError();
}

int refshim_diff2_coarse_double(void* h, int imgX, int imgY, int imgZ,
                                int imgMaxR, float* d_eulers, float* d_tx,
                                float* d_ty, float* d_corr, float* d_re,
                                float* d_im, double* d_diff2s, long O, long T,
                                long N_img, int filter_img, void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  runDiff2KernelCoarseDouble(k, d_tx, d_ty, nullptr, d_corr, d_re, d_im,
                             d_eulers, d_diff2s, 1.f, (unsigned long)O,
                             (unsigned long)T, (unsigned long)N_img,
                             (cudaStream_t)stream, false, false,
                             filter_img != 0);
  return (int)cudaGetLastError();
}

// variant: 0 cuda-core im2col, 1 tensor-core im2col, 2 + conflict removal,
// 3 + texture-fetch masking (filtered image), 4 + cross-CTA translation reuse
// (filtered image, workspace).  Constructor arguments follow the functors'
// declared meaning (T, O, image_size, full_image_size, sm_num); the harness at
// src/main.cu:399-411 passes sm_num into full_image_size for variants 0-2.
size_t refshim_variant_workspace_bytes(int variant, int T, int O, int K_filtered,
                                       int N_img, int sm_num) {
  if (variant == 4) {
    CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse<> k(
        T, O, K_filtered, N_img, sm_num);
    return k.get_workspace_size_bytes();
  }
  return 0;
}

int refshim_variant_run(int variant, void* h, int imgX, int imgY, int imgZ,
                        int imgMaxR, float* d_eulers, float* d_tx, float* d_ty,
                        float* d_re, float* d_im, float* d_corr,
                        float* d_diff2s, float* d_coor_xy,
                        unsigned int* d_workspace, int T, int O, int K_filtered,
                        int N_img, int sm_num, void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  cudaStream_t s = (cudaStream_t)stream;
  switch (variant) {
    case 0: {
      CoarseMatrixKernelCudaCoreIm2colSplitImgNfuse<> f(T, O, N_img, 0, sm_num);
      f.run(d_eulers, d_tx, d_ty, d_re, d_im, k, d_corr, d_diff2s, d_diff2s, s);
      break;
    }
    case 1: {
      CoarseMatrixKernelIm2colSplitImgNfuse<> f(T, O, N_img, 0, sm_num);
      f.run(d_eulers, d_tx, d_ty, d_re, d_im, k, d_corr, d_diff2s, d_diff2s, s);
      break;
    }
    case 2: {
      CoarseMatrixKernelIm2colSplitImgBCFNfuse<> f(T, O, N_img, 0, sm_num);
      f.run(d_eulers, d_tx, d_ty, d_re, d_im, k, d_corr, d_diff2s, d_diff2s, s);
      break;
    }
    case 3: {
      CoarseMatrixKernelIm2colSplitImgBCFProjOverlapNfuse<> f(
          T, O, K_filtered, N_img, sm_num);
      f.run(d_eulers, d_tx, d_ty, d_re, d_im, k, d_corr, d_diff2s, d_diff2s, s,
            d_coor_xy);
      break;
    }
    case 4: {
      CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse<> f(
          T, O, K_filtered, N_img, sm_num);
      f.run(d_eulers, d_tx, d_ty, d_re, d_im, k, d_corr, d_diff2s, d_diff2s, s,
            d_coor_xy, d_workspace);
      break;
    }
    default:
      return -1;
  }
  return (int)cudaGetLastError();
}

// The fine-pass kernel has no host wrapper in the reference; this launches
// it for a 3D reference and 2D images with 128-thread blocks and up to 16
// translations per job (its shared-memory buffer is block_sz * chunk_sz).
int refshim_diff2_fine(void* h, int imgX, int imgY, int imgZ, int imgMaxR, float* d_eulers, float* d_re,
                       float* d_im, float* d_tx, float* d_ty, float* d_corr, float* d_diff2s, long image_size,
                       float sum_init, long O, long T, long todo_blocks, unsigned long* d_rot_idx,
                       unsigned long* d_trans_idx, unsigned long* d_job_idx, unsigned long* d_job_num,
                       void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  cuda_kernel_diff2_fine<true, false, 128, 16><<<(unsigned)todo_blocks, 128, 0, (cudaStream_t)stream>>>(
      d_eulers, d_re, d_im, d_tx, d_ty, nullptr, k, d_corr, d_diff2s, (unsigned)image_size, sum_init,
      (unsigned long)O, (unsigned long)T, (unsigned long)todo_blocks, d_rot_idx, d_trans_idx, d_job_idx, d_job_num);
  return (int)cudaGetLastError();
}

// The CC form, launched the same way (sum_init and exp_local_sqrtXi2 are not
// read by the kernel).
int refshim_diff2_fine_cc(void* h, int imgX, int imgY, int imgZ, int imgMaxR, float* d_eulers, float* d_re,
                          float* d_im, float* d_tx, float* d_ty, float* d_corr, float* d_diff2s, long image_size,
                          long O, long T, long todo_blocks, unsigned long* d_rot_idx, unsigned long* d_trans_idx,
                          unsigned long* d_job_idx, unsigned long* d_job_num, void* stream) {
  RefProjector* p = reinterpret_cast<RefProjector*>(h);
  AccProjectorKernel k = make_view(p, imgX, imgY, imgZ, imgMaxR);
  cuda_kernel_diff2_CC_fine<true, false, 128, 16><<<(unsigned)todo_blocks, 128, 0, (cudaStream_t)stream>>>(
      d_eulers, d_re, d_im, d_tx, d_ty, nullptr, k, d_corr, d_diff2s, (unsigned)image_size, 0.f, 1.f,
      (unsigned long)O, (unsigned long)T, (unsigned long)todo_blocks, d_rot_idx, d_trans_idx, d_job_idx, d_job_num);
  return (int)cudaGetLastError();
}

// The significance kernels, launched the way RELION's host helpers
// (findThresholdIdxInCumulativeSum, arrayOverThreshold) do: a grid over the
// array, the index word cleared first; block size 256.
int refshim_find_threshold_idx(double* d_cum, double thr, long size, unsigned long* d_idx, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(d_idx, 0, sizeof(size_t), s);
  if (e != cudaSuccess) return (int)e;
  const int bs = 256;
  const long grid = size > 1 ? (size - 1 + bs - 1) / bs : 0;
  if (grid == 0) return 0;
  cuda_kernel_find_threshold_idx_in_cumulative<double><<<(unsigned)grid, bs, 0, s>>>(
      d_cum, thr, (size_t)(size - 1), reinterpret_cast<size_t*>(d_idx), bs);
  return (int)cudaGetLastError();
}

int refshim_array_over_threshold(double* d_data, bool* d_passed, double thr, long size, void* stream) {
  const int bs = 256;
  const long grid = (size + bs - 1) / bs;
  if (grid == 0) return 0;
  cuda_kernel_array_over_threshold<double><<<(unsigned)grid, bs, 0, (cudaStream_t)stream>>>(
      d_data, d_passed, thr, (size_t)size, bs);
  return (int)cudaGetLastError();
}

}  // extern "C"
