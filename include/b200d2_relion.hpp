// b200d2_relion.hpp -- the reference harness's C++ API on top of the C ABI.
//
// A caller written against Edgarrrrrr/T2-RELION-kernel includes this header
// instead of the reference headers and links libb200d2.so.  Same class and
// function names, argument lists and semantics as:
//   AccProjector                src/acc_projector.h:12-86, src/acc_projector_impl.h
//   AccProjectorKernel          src/acc_projectorkernel_impl.h:15-60, makeKernel :410-433
//   runDiff2KernelCoarse        src/acc_helper_functions_impl.h:15-31
//   runDiff2KernelCoarseDouble  src/acc_helper_functions_impl.h:503-520
//   CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse
//                               src/coarse_splitImg_BCF_PMO_TMDB_NFUSE.cuh:40-131
// Differences a caller may notice:
//   * errors throw b200d2_relion_error (the reference raises SIGSEGV through
//     HANDLE_ERROR, src/common.h:20-36);
//   * do_CC runs the CC score (b200d2_diff2_coarse_cc); the data_is_3D
//     branches are not provided (they throw);
//   * the optimised functor runs the tensor-core pipeline (BF16 3-term split
//     by default, B200D2_RELION_FUNCTOR_PRECISION to change) and its
//     workspace needs no 0xff pre-fill.
#ifndef B200D2_RELION_HPP_
#define B200D2_RELION_HPP_

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

#include "b200d2.h"

#ifndef XFLOAT
#define XFLOAT float
#endif

#ifndef B200D2_RELION_FUNCTOR_PRECISION
#define B200D2_RELION_FUNCTOR_PRECISION B200D2_PREC_BF16X3
#endif

struct b200d2_relion_error : std::runtime_error {
  int status;
  b200d2_relion_error(const std::string& w, int s)
      : std::runtime_error(w + ": b200d2 status " + std::to_string(s)), status(s) {}
};

namespace b200d2_relion_detail {
inline void check(int st, const char* where) {
  if (st != B200D2_OK) throw b200d2_relion_error(where, st);
}
}  // namespace b200d2_relion_detail

class AccProjectorKernel;

class AccProjector {
  friend class AccProjectorKernel;
  int mdlX = 0, mdlY = 0, mdlZ = 0, mdlMaxR = 0, mdlInitY = 0, mdlInitZ = 0;
  XFLOAT padding_factor = 0;
  size_t mdlXYZ = 0;
  b200d2_projector* handle_ = nullptr;

 public:
  AccProjector() = default;
  AccProjector(const AccProjector&) = delete;
  AccProjector& operator=(const AccProjector&) = delete;
  ~AccProjector() { clear(); }

  // Records the model geometry; returns false if it is unchanged.
  bool setMdlDim(int xdim, int ydim, int zdim, int inity, int initz, int maxr, XFLOAT paddingFactor) {
    if (zdim == 1) zdim = 0;
    if (xdim == mdlX && ydim == mdlY && zdim == mdlZ && inity == mdlInitY && initz == mdlInitZ &&
        maxr == mdlMaxR && paddingFactor == padding_factor)
      return false;
    clear();
    mdlX = xdim;
    mdlY = ydim;
    mdlZ = zdim;
    mdlXYZ = (size_t)xdim * ydim * (zdim == 0 ? 1 : zdim);
    mdlInitY = inity;
    mdlInitZ = initz;
    mdlMaxR = maxr;
    padding_factor = paddingFactor;
    return true;
  }

  // Uploads the volume (host arrays, copied) into texture arrays.
  void initMdl(XFLOAT* real, XFLOAT* imag) {
    if (handle_) b200d2_projector_destroy(handle_);
    handle_ = nullptr;
#ifdef PROJECTOR_NO_TEXTURES
    const int rep = 0;
#else
    const int rep = 1;
#endif
    b200d2_relion_detail::check(b200d2_projector_create(mdlX, mdlY, mdlZ, mdlInitY, mdlInitZ, mdlMaxR,
                                                        padding_factor, real, imag, rep, &handle_),
                                "AccProjector::initMdl");
  }

  void clear() {
    if (handle_) b200d2_projector_destroy(handle_);
    handle_ = nullptr;
  }

  void constructFromFile(const std::string& filename) {
    clear();
#ifdef PROJECTOR_NO_TEXTURES
    const int rep = 0;
#else
    const int rep = 1;
#endif
    b200d2_relion_detail::check(b200d2_projector_load_dat(filename.c_str(), rep, &handle_),
                                "AccProjector::constructFromFile");
    int d[6];
    float pf = 0.f;
    b200d2_relion_detail::check(b200d2_projector_dims(handle_, d, &pf), "AccProjector::constructFromFile");
    mdlX = d[0];
    mdlY = d[1];
    mdlZ = d[2];
    mdlInitY = d[3];
    mdlInitZ = d[4];
    mdlMaxR = d[5];
    padding_factor = pf;
    mdlXYZ = (size_t)mdlX * mdlY * (mdlZ == 0 ? 1 : mdlZ);
  }

  const b200d2_projector* handle() const { return handle_; }
};

class AccProjectorKernel {
 public:
  int mdlX = 0, mdlXY = 0, mdlZ = 0, imgX = 0, imgY = 0, imgZ = 0, mdlInitY = 0, mdlInitZ = 0, maxR = 0,
      maxR2 = 0, maxR2_padded = 0;
  XFLOAT padding_factor = 0;
  b200d2_view view{};

  static AccProjectorKernel makeKernel(AccProjector& p, int imgX, int imgY, int imgZ, int imgMaxR) {
    AccProjectorKernel k;
#ifdef PROJECTOR_NO_TEXTURES
    const int interp = B200D2_INTERP_LINEAR;
#else
    const int interp = B200D2_INTERP_TEXTURE;
#endif
    b200d2_relion_detail::check(b200d2_projector_view(p.handle_, imgX, imgY, imgZ, imgMaxR, interp, &k.view),
                                "AccProjectorKernel::makeKernel");
    k.mdlX = k.view.mdlX;
    k.mdlXY = k.view.mdlXY;
    k.mdlZ = k.view.mdlZ;
    k.imgX = k.view.imgX;
    k.imgY = k.view.imgY;
    k.imgZ = k.view.imgZ;
    k.mdlInitY = k.view.mdlInitY;
    k.mdlInitZ = k.view.mdlInitZ;
    k.maxR = k.view.maxR;
    k.maxR2 = k.view.maxR2;
    k.maxR2_padded = k.view.maxR2_padded;
    k.padding_factor = k.view.padding_factor;
    return k;
  }
};

// Precision of runDiff2KernelCoarse's non-CC branch, process-wide:
// B200D2_PREC_FP32 (default: FP32 CUDA cores, within 1e-5 of the reference's
// own kernel) or a tensor-core precision (the one-particle tensor-core
// pipeline on a library-owned workspace; B200D2_PREC_BF16X3 stays within 1e-5
// of the FP64 kernel).  Returns the previous setting.
inline int setCoarsePrecision(int precision) {
  static int p = B200D2_PREC_FP32;
  const int old = p;
  if (precision >= 0) p = precision;
  return old;
}
inline int coarsePrecision() {
  const int p = setCoarsePrecision(-1);
  return p;
}

// diff2s[o*T + t] += diff2(o, t)  (asynchronous on `stream`, in the precision
// set by setCoarsePrecision); with do_CC, diff2s[o*T + t] = -cross / sqrt(norm)
// as cuda_kernel_diff2_CC_coarse (src/diff2.cuh:691-809) writes it.
inline void runDiff2KernelCoarse(AccProjectorKernel& projector, XFLOAT* trans_x, XFLOAT* trans_y,
                                 XFLOAT* /*trans_z*/, XFLOAT* corr_img, XFLOAT* Fimg_real, XFLOAT* Fimg_imag,
                                 XFLOAT* d_eulers, XFLOAT* diff2s, XFLOAT /*local_sqrtXi2*/,
                                 unsigned long orientation_num, unsigned long translation_num,
                                 unsigned long image_size, cudaStream_t stream, bool do_CC, bool data_is_3D) {
  if (data_is_3D) throw b200d2_relion_error("runDiff2KernelCoarse: data_is_3D", B200D2_ERR_UNSUPPORTED);
  if (do_CC) {
    b200d2_relion_detail::check(
        b200d2_diff2_coarse_cc(&projector.view, trans_x, trans_y, corr_img, Fimg_real, Fimg_imag, d_eulers, diff2s,
                               orientation_num, translation_num, image_size, stream, B200D2_PREC_FP32),
        "runDiff2KernelCoarse(do_CC)");
    return;
  }
  b200d2_relion_detail::check(
      b200d2_diff2_coarse(&projector.view, trans_x, trans_y, corr_img, Fimg_real, Fimg_imag, d_eulers, diff2s,
                          orientation_num, translation_num, image_size, stream, coarsePrecision()),
      "runDiff2KernelCoarse");
}

inline void runDiff2KernelCoarseDouble(AccProjectorKernel& projector, XFLOAT* trans_x, XFLOAT* trans_y,
                                       XFLOAT* /*trans_z*/, XFLOAT* corr_img, XFLOAT* Fimg_real,
                                       XFLOAT* Fimg_imag, XFLOAT* d_eulers, double* diff2s,
                                       XFLOAT /*local_sqrtXi2*/, unsigned long orientation_num,
                                       unsigned long translation_num, unsigned long image_size,
                                       cudaStream_t stream, bool do_CC, bool data_is_3D, bool filter_img = false) {
  // the reference's FP64 dispatcher has no CC branch: do_CC is ignored there
  // (src/acc_helper_functions_impl.h:503-854), and here
  (void)do_CC;
  if (data_is_3D) throw b200d2_relion_error("runDiff2KernelCoarseDouble: data_is_3D", B200D2_ERR_UNSUPPORTED);
  b200d2_relion_detail::check(
      b200d2_diff2_coarse_f64(&projector.view, trans_x, trans_y, corr_img, Fimg_real, Fimg_imag, d_eulers,
                              diff2s, orientation_num, translation_num, image_size, filter_img ? 1 : 0, stream),
      "runDiff2KernelCoarseDouble");
}

// The reference's best optimised functor, same constructor and run()
// arguments.  image_size is the number of filtered (in-radius) pixels,
// full_image_size the total; the image arrays are in the filtered order and
// g_coor_xy holds the (x, y) of the filtered pixels (required, as the
// reference harness always passes it for this functor, src/main.cu:418-421).
// Accumulates into g_diff2s_dest (which, as in the reference, should equal
// g_diff2s).
template <typename TParams = void>
struct CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse {
  const int translation_num_;
  const int orientation_num_;
  const int image_size_;
  const int full_image_size_;
  const int sm_num_;

  CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse(int translation_num, int orientation_num,
                                                             int image_size, int full_image_size,
                                                             int sm_num = 108)
      : translation_num_(translation_num),
        orientation_num_(orientation_num),
        image_size_(image_size),
        full_image_size_(full_image_size),
        sm_num_(sm_num) {}

  b200d2_batch batch_(XFLOAT* eul, XFLOAT* tx, XFLOAT* ty, XFLOAT* re, XFLOAT* im, XFLOAT* corr, XFLOAT* dst,
                      XFLOAT* coor_xy) const {
    b200d2_batch b{};
    b.d_eulers = eul;
    b.O = orientation_num_;
    b.d_trans_x = tx;
    b.d_trans_y = ty;
    b.T = translation_num_;
    b.P = 1;
    b.N_img = full_image_size_ > image_size_ ? full_image_size_ : image_size_;
    b.d_real = re;
    b.d_imag = im;
    b.d_corr = corr;
    b.img_stride = b.N_img;
    b.d_diff2 = dst;
    b.accumulate = 1;
    b.d_coor_xy = coor_xy;
    b.n_listed = coor_xy ? image_size_ : 0;
    return b;
  }

  // Workspace bytes for this shape (independent of the projector contents).
  size_t get_workspace_size_bytes() const {
    b200d2_view v{};
    v.mdlX = v.mdlXY = v.mdlZ = 1;
    v.imgX = 32767;
    v.imgY = 32767;
    v.interp = B200D2_INTERP_LINEAR;
    v.lin_re = v.lin_im = reinterpret_cast<const float*>(16);
    v.maxR = 512;
    v.padding_factor = 1.f;
    float dummy = 0.f;
    b200d2_batch b = batch_(&dummy, &dummy, &dummy, &dummy, &dummy, &dummy, &dummy, &dummy);
    return b200d2_diff2_coarse_batch_workspace(&v, &b, B200D2_RELION_FUNCTOR_PRECISION);
  }

  void run(XFLOAT* g_eulers, XFLOAT* trans_x, XFLOAT* trans_y, XFLOAT* g_real, XFLOAT* g_imag,
           AccProjectorKernel projector, XFLOAT* g_corr, XFLOAT* g_diff2s, XFLOAT* g_diff2s_dest,
           cudaStream_t stream, XFLOAT* g_coor_xy = nullptr, uint32_t* work_space = nullptr) {
    if (!g_coor_xy || !work_space)
      throw b200d2_relion_error("CoarseMatrixKernel::run needs g_coor_xy and work_space", B200D2_ERR_INVALID);
    if (g_diff2s != g_diff2s_dest)
      b200d2_relion_detail::check(
          cudaMemcpyAsync(g_diff2s_dest, g_diff2s,
                          sizeof(XFLOAT) * (size_t)orientation_num_ * translation_num_, cudaMemcpyDeviceToDevice,
                          stream) == cudaSuccess
              ? B200D2_OK
              : B200D2_ERR_CUDA,
          "CoarseMatrixKernel::run");
    b200d2_batch b = batch_(g_eulers, trans_x, trans_y, g_real, g_imag, g_corr, g_diff2s_dest, g_coor_xy);
    const size_t need = get_workspace_size_bytes();
    b200d2_relion_detail::check(b200d2_diff2_coarse_batch(&projector.view, &b, B200D2_RELION_FUNCTOR_PRECISION,
                                                          work_space, need, stream),
                                "CoarseMatrixKernel::run");
  }
};

#endif  // B200D2_RELION_HPP_
