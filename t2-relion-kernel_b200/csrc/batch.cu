// batch.cu -- the batched coarse pass entry (b200d2_diff2_coarse_batch).
//
// Dispatches on precision: the CUDA-core direct kernels (FP32, FP64) or the
// tensor-core pipeline (tc_pipeline.cu).  The reference has no batched call:
// its harness loops runDiff2KernelCoarse over particles (src/main.cu:483-503).
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace b200d2 {
int direct_batch(const b200d2_view& view, const float* eulers, const float* tx,
                 const float* ty, const float* re, const float* im,
                 const float* corr, long long img_stride, void* out,
                 long long out_stride, int O, int T, int N_img, int P,
                 bool fp64, int filter_img, cudaStream_t s, int cc, int accumulate);
int minloc(const float* d, long long n, int P, double* mn, long long* arg, cudaStream_t s);
size_t tc_workspace_bytes(const b200d2_view& view, const b200d2_batch& b, int precision,
                          bool allow_split = true);
int tc_run(const b200d2_view& view, const b200d2_batch& b, int precision, void* ws,
           size_t ws_bytes, cudaStream_t s, const int* d_proj_need = nullptr,
           float* d_eul_cache = nullptr);
bool tc_projection_layout(const b200d2_view& v, const b200d2_batch& b, int precision, std::vector<uint64_t>& key);

static int validate(const b200d2_view* v, const b200d2_batch* b) {
  if (!v || !b) return B200D2_ERR_INVALID;
  if (b->O < 0 || b->T < 0 || b->P < 0 || b->N_img < 0) return B200D2_ERR_INVALID;
  if (b->O == 0 || b->T == 0 || b->P == 0) return B200D2_OK;
  if (!b->d_eulers || !b->d_trans_x || !b->d_trans_y || !b->d_real || !b->d_imag ||
      !b->d_corr || !b->d_diff2)
    return B200D2_ERR_INVALID;
  if (b->img_stride < b->N_img) return B200D2_ERR_INVALID;
  if ((long long)v->imgX * v->imgY < b->N_img) return B200D2_ERR_INVALID;
  if (v->mdlZ == 0) return B200D2_ERR_UNSUPPORTED;
  if (v->interp == B200D2_INTERP_TEXTURE && (!v->tex_re || !v->tex_im)) return B200D2_ERR_INVALID;
  if (v->interp == B200D2_INTERP_LINEAR && (!v->lin_re || !v->lin_im)) return B200D2_ERR_INVALID;
  if (v->imgX > 32767 || v->imgY > 32767) return B200D2_ERR_UNSUPPORTED;
  if (b->d_coor_xy && (b->n_listed < 0 || b->n_listed > b->N_img)) return B200D2_ERR_INVALID;
  if (b->score != B200D2_SCORE_DIFF2 && b->score != B200D2_SCORE_CC) return B200D2_ERR_INVALID;
  return B200D2_OK;
}

static unsigned long long g_launches = 0;
void count_launch(unsigned n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
unsigned long long launch_counter() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
void uncount_launch(unsigned n) { __atomic_fetch_sub(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }

// Workspaces owned by the library for the single-particle entry point with a
// tensor-core precision, whose signature (runDiff2KernelCoarse's) carries
// none: one per (device, stream), allocated and grown stream-ordered
// (cudaMallocAsync / cudaFreeAsync on that stream, so calls queued on the
// stream before the growth finish with the old buffer), kept until the
// process exits.
//
// Projection cache.  A caller of the single-particle signature scores one
// particle after another against the same orientations (the reference's
// harness loops runDiff2KernelCoarse over particles with one Euler array,
// src/main.cu:483-503), and the projections of those orientations are most
// of a call's work.  The workspace keeps the last call's projections; the
// next call skips its projection stage when
//   - everything the projections and their place in the workspace depend on,
//     other than the Euler matrices, is unchanged (host key: the view, the
//     workspace address and layout, the precision, the projector epoch,
//     which advances whenever any projector is created or destroyed), and
//   - its Euler matrices equal, bit for bit, those of the call that projected
//     (compared on the device against a copy kept with the workspace, so the
//     check needs no host synchronisation and sees contents changed in place).
// Otherwise it projects and the projection stage refreshes the copy.  Skipped
// or not, the scores are bit-identical.  The FP16 forms, whose projection
// stage rescales per call, and projections of fewer than 2^20 samples (faster
// than the check) always project.
struct OwnedWorkspace {
  int device;
  cudaStream_t stream;
  void* ptr;
  size_t bytes;
  float* eul;                 // device copy of the Euler matrices last projected, then the verdict words
  size_t eul_cap;             // floats
  int* need;                  // device: kEulCheckBlocks verdict words, any nonzero = project this call
  std::vector<uint64_t> key;  // host key of the cached projections; empty = none
};
static std::mutex g_owned_mu;
static std::vector<OwnedWorkspace> g_owned;
static std::atomic<int> g_proj_cache{1};  // b200d2_set_projection_cache

// (with g_owned_mu held)
static int owned_workspace(cudaStream_t s, size_t need, OwnedWorkspace** out) {
  int dev = 0;
  B200D2_CUDA_TRY(cudaGetDevice(&dev));
  for (OwnedWorkspace& w : g_owned)
    if (w.device == dev && w.stream == s) {
      if (w.bytes < need) {
        w.key.clear();
        B200D2_CUDA_TRY(cudaFreeAsync(w.ptr, s));
        w.ptr = nullptr;
        w.bytes = 0;
        B200D2_CUDA_TRY(cudaMallocAsync(&w.ptr, need, s));
        w.bytes = need;
      }
      *out = &w;
      return B200D2_OK;
    }
  OwnedWorkspace w{dev, s, nullptr, need, nullptr, 0, nullptr, {}};
  B200D2_CUDA_TRY(cudaMallocAsync(&w.ptr, need, s));
  g_owned.push_back(w);
  *out = &g_owned.back();
  return B200D2_OK;
}

// need[b] = force, or whether any Euler value of block b's share differs
// (bit for bit) from the copy of the last projected ones; every word is
// written each call, so none needs a reset.  The projection stage ORs the
// kEulCheckBlocks words and, when it projects, refreshes the copy.
__global__ void __launch_bounds__(256) eul_check_kernel(const float* __restrict__ a,
                                                        const float* __restrict__ cached, int n, int force,
                                                        int* need) {
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  int differ = force;
  if (!force)
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x)
      differ |= __float_as_uint(a[i]) != __float_as_uint(cached[i]);
  differ = __syncthreads_or(differ);
  if (threadIdx.x == 0) need[blockIdx.x] = differ;
}

// One particle through the tensor-core pipeline, accumulating onto diff2s as
// the reference's runDiff2KernelCoarse does.
int single_particle_tc(const b200d2_view& v, const float* tx, const float* ty, const float* corr, const float* re,
                       const float* im, const float* eulers, float* diff2s, int O, int T, int N_img, int precision,
                       cudaStream_t s) {
  b200d2_batch b;
  memset(&b, 0, sizeof(b));
  b.d_eulers = eulers;
  b.O = O;
  b.d_trans_x = tx;
  b.d_trans_y = ty;
  b.T = T;
  b.P = 1;
  b.N_img = N_img;
  b.d_real = re;
  b.d_imag = im;
  b.d_corr = corr;
  b.img_stride = N_img;
  b.d_diff2 = diff2s;
  b.accumulate = 1;
  int st = validate(&v, &b);
  if (st != B200D2_OK) return st;
  const size_t need = tc_workspace_bytes(v, b, precision);
  std::vector<uint64_t> key;
  const bool cacheable = g_proj_cache.load() != 0 && tc_projection_layout(v, b, precision, key);
  std::lock_guard<std::mutex> lk(g_owned_mu);
  OwnedWorkspace* w = nullptr;
  st = owned_workspace(s, need, &w);
  if (st != B200D2_OK) return st;
  if (!cacheable) {
    w->key.clear();
    return tc_run(v, b, precision, w->ptr, need, s);
  }
  uint32_t pf;
  memcpy(&pf, &v.padding_factor, 4);
  key.insert(key.end(), {(uint64_t)v.mdlX, (uint64_t)v.mdlXY, (uint64_t)v.mdlZ, (uint64_t)v.imgX, (uint64_t)v.imgY,
                         (uint64_t)v.imgZ, (uint64_t)(uint32_t)v.mdlInitY, (uint64_t)(uint32_t)v.mdlInitZ,
                         (uint64_t)v.maxR, (uint64_t)v.maxR2, (uint64_t)v.maxR2_padded, (uint64_t)pf, v.tex_re,
                         v.tex_im, (uint64_t)(uintptr_t)v.lin_re, (uint64_t)(uintptr_t)v.lin_im,
                         (uint64_t)v.interp, v.tex_c, projector_epoch(), (uint64_t)(uintptr_t)w->ptr,
                         (uint64_t)N_img});
  const int n = O * 9;
  if (w->eul_cap < (size_t)n) {
    w->key.clear();
    if (w->eul) B200D2_CUDA_TRY(cudaFreeAsync(w->eul, s));
    w->eul = nullptr;
    w->eul_cap = 0;
    const size_t at = ((size_t)n * sizeof(float) + 15) / 16 * 16;
    void* p = nullptr;
    B200D2_CUDA_TRY(cudaMallocAsync(&p, at + sizeof(int) * kEulCheckBlocks, s));
    w->eul = static_cast<float*>(p);
    w->need = reinterpret_cast<int*>(static_cast<char*>(p) + at);
    w->eul_cap = (size_t)n;
  }
  const bool force = key != w->key;
  w->key.clear();  // set again once this call's launches are issued
  eul_check_kernel<<<kEulCheckBlocks, 256, 0, s>>>(eulers, w->eul, n, force ? 1 : 0, w->need);
  count_launch();
  B200D2_CUDA_TRY(cudaGetLastError());
  st = tc_run(v, b, precision, w->ptr, need, s, w->need, w->eul);
  if (st == B200D2_OK) w->key = key;
  return st;
}

}  // namespace b200d2

extern "C" int b200d2_set_projection_cache(int enable) {
  if (enable != 0 && enable != 1) return B200D2_ERR_INVALID;
  b200d2::g_proj_cache.store(enable);
  return B200D2_OK;
}

extern "C" unsigned long long b200d2_launch_count(void) {
  return __atomic_load_n(&b200d2::g_launches, __ATOMIC_RELAXED);
}

extern "C" size_t b200d2_diff2_coarse_batch_workspace(const b200d2_view* view,
                                                      const b200d2_batch* batch,
                                                      int precision) {
  if (b200d2::validate(view, batch) != B200D2_OK) return 0;
  if (precision == B200D2_PREC_FP32 || precision == B200D2_PREC_FP64) return 0;
  return b200d2::tc_workspace_bytes(*view, *batch, precision);
}

extern "C" int b200d2_diff2_coarse_batch(const b200d2_view* view, const b200d2_batch* batch,
                                         int precision, void* d_workspace,
                                         size_t workspace_bytes, void* stream) {
  int st = b200d2::validate(view, batch);
  if (st != B200D2_OK) return st;
  const b200d2_batch& b = *batch;
  if (b.d_coor_xy && (precision == B200D2_PREC_FP32 || precision == B200D2_PREC_FP64))
    return B200D2_ERR_UNSUPPORTED;  // listed pixels: tensor-core path only
  if (b.O == 0 || b.T == 0 || b.P == 0) return B200D2_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long per = (long long)b.O * b.T;
  if (precision == B200D2_PREC_FP32) {
    const int cc = b.score == B200D2_SCORE_CC;
    if (!b.accumulate && !cc)  // the diff2 kernel adds; the CC kernel writes unless told to add
      B200D2_CUDA_TRY(cudaMemsetAsync(b.d_diff2, 0, sizeof(float) * per * b.P, s));
    st = b200d2::direct_batch(*view, b.d_eulers, b.d_trans_x, b.d_trans_y, b.d_real, b.d_imag,
                              b.d_corr, b.img_stride, b.d_diff2, per, b.O, b.T, b.N_img, b.P,
                              false, 0, s, cc, b.accumulate);
    if (st != B200D2_OK) return st;
    if (b.d_min || b.d_argmin) st = b200d2::minloc(b.d_diff2, per, b.P, b.d_min, b.d_argmin, s);
    return st;
  }
  if (b200d2::is_tc_precision(precision)) {
    const size_t need = b200d2::tc_workspace_bytes(*view, b, precision);
    if (need > 0 && (!d_workspace || workspace_bytes < need)) return B200D2_ERR_INVALID;
    return b200d2::tc_run(*view, b, precision, d_workspace, workspace_bytes, s);
  }
  return B200D2_ERR_UNSUPPORTED;
}

namespace b200d2 {
const char* tc_stage_name(int precision, int stage);
int tc_run_stage(const b200d2_view& view, const b200d2_batch& b, int precision, int stage,
                 void* ws, size_t ws_bytes, cudaStream_t s, bool allow_split = true);
}  // namespace b200d2

extern "C" const char* b200d2_stage_name(int precision, int stage) {
  if (precision == B200D2_PREC_FP32) {
    static const char* names[] = {"diff2_direct_kernel<float>", "minloc_kernel"};
    return (stage >= 0 && stage < 2) ? names[stage] : nullptr;
  }
  if (b200d2::is_tc_precision(precision))
    return b200d2::tc_stage_name(precision, stage);
  return nullptr;
}

extern "C" int b200d2_diff2_coarse_batch_stage(const b200d2_view* view,
                                               const b200d2_batch* batch, int precision,
                                               int stage, void* d_workspace,
                                               size_t workspace_bytes, void* stream) {
  int st = b200d2::validate(view, batch);
  if (st != B200D2_OK) return st;
  const b200d2_batch& b = *batch;
  if (b.d_coor_xy && (precision == B200D2_PREC_FP32 || precision == B200D2_PREC_FP64))
    return B200D2_ERR_UNSUPPORTED;  // listed pixels: tensor-core path only
  if (b.O == 0 || b.T == 0 || b.P == 0) return B200D2_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long per = (long long)b.O * b.T;
  if (precision == B200D2_PREC_FP32) {
    if (stage == 0)
      return b200d2::direct_batch(*view, b.d_eulers, b.d_trans_x, b.d_trans_y, b.d_real,
                                  b.d_imag, b.d_corr, b.img_stride, b.d_diff2, per, b.O, b.T,
                                  b.N_img, b.P, false, 0, s, b.score == B200D2_SCORE_CC, 1);
    if (stage == 1) return b200d2::minloc(b.d_diff2, per, b.P, b.d_min, b.d_argmin, s);
    return B200D2_ERR_INVALID;
  }
  if (b200d2::is_tc_precision(precision)) {
    const size_t need = b200d2::tc_workspace_bytes(*view, b, precision);
    if (need > 0 && (!d_workspace || workspace_bytes < need)) return B200D2_ERR_INVALID;
    return b200d2::tc_run_stage(*view, b, precision, stage, d_workspace, workspace_bytes, s);
  }
  return B200D2_ERR_UNSUPPORTED;
}
