// fine.cu -- fine-pass diff2 over a job list (b200d2_diff2_fine).
//
// Replaces cuda_kernel_diff2_fine (src/diff2.cuh:540-682, 2D image against a
// 3D reference).  After the coarse pass, RELION rescores only the significant
// samples on oversampled orientation and translation grids.  The work arrives
// as jobs: job j scores orientation rot_idx[job_idx[j]] against the job_num[j]
// consecutive translations starting at trans_idx[job_idx[j]], and writes
//   diff2s[job_idx[j] + i] = sum_init + sum_px corr/2 |proj - shift_i(img)|^2
// for i < job_num[j] (written, not accumulated, as the reference does).
//
// One CTA per job.  Each thread projects its pixels once (texture or linear
// projector, the same sample positions as the coarse kernels) and keeps the
// job's translations in registers (up to kFineMaxTrans per pass; longer jobs
// take several passes over the pixels), so the projection is shared by all of
// the job's translations; the per-translation sums are reduced with warp
// shuffles and one shared-memory step in a fixed order.  The phase shift
// e^{i(x tx + y ty)} is the product of two table entries e^{i x tx} and
// e^{i y ty}, built per pass in shared memory (one sincos per table entry,
// not per pixel).  With the tables the score is taken expanded,
//   sum w|A - S|^2 = sum w(|A|^2 + |X|^2) - 2 sum Re(q e^{i x tx} e^{i y ty}),
//   q = w conj(A) X,
// so a (pixel, translation) pair costs one complex multiply and a real part
// (the norms are per pixel, in FP64); the per-thread cross sums are combined
// in FP64 and the final difference is taken in FP64.  Jobs on images too
// large for the tables take sincosf per pixel and sum w|A - S|^2 directly, as
// the reference does.  Pixel coordinates
// follow the fine kernel's mapping (src/diff2.cuh:612-626): rows past maxR
// wrap to negative y when they lie within maxR of the end, otherwise their x
// is set to maxR (outside the projector radius).
//
// The same kernel with CC = true replaces cuda_kernel_diff2_CC_fine
// (src/diff2.cuh:811-960): per (job, translation) it writes
//   diff2s[job_idx[j] + i] = -sum_px corr Re(conj(proj) shift_i(img)) / sqrt(sum_px corr |proj|^2)
// (full corr, no sum_init, written).  The cross sums are taken as above with
// q = corr conj(A) X; the norm is summed in FP64 and the quotient taken in
// FP64.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace b200d2 {

constexpr int kFineThreads = 128;
constexpr int kFineMaxTrans = 16;
constexpr size_t kFineTableBytes = 96 * 1024;  // largest phase-table area per CTA

__device__ __forceinline__ void fine_pixel_coor(int pixel, int imgX, int imgY, int maxR, int& x, int& y) {
  x = pixel % imgX;
  y = pixel / imgX;
  if (y > maxR) {
    if (y >= imgY - maxR)
      y -= imgY;
    else
      x = maxR;
  }
}

template <int NT, bool TABLES, bool CC>
__global__ void __launch_bounds__(kFineThreads) diff2_fine_kernel(
    b200d2_view v, const float* __restrict__ eulers, const float* __restrict__ re, const float* __restrict__ im,
    const float* __restrict__ tx, const float* __restrict__ ty, const float* __restrict__ corr,
    float* __restrict__ diff2s, int image_size, float sum_init, const uint64_t* __restrict__ rot_idx,
    const uint64_t* __restrict__ trans_idx, const uint64_t* __restrict__ job_idx,
    const uint64_t* __restrict__ job_num) {
  const uint64_t jb = job_idx[blockIdx.x];
  const int ntrans = (int)job_num[blockIdx.x];
  const uint64_t o = rot_idx[jb];
  const uint64_t t0 = trans_idx[jb];
  const float* eo = eulers + o * 9;
  float e[6] = {eo[0], eo[1], eo[3], eo[4], eo[6], eo[7]};
  __shared__ float s_part[kFineThreads / 32][NT];
  __shared__ double s_cross[kFineThreads / 32][NT], s_norm[kFineThreads / 32];
  // TABLES: [NT][exw] e^{i x tx} for x in [0, exw), then [NT][eyw] e^{i y ty}
  // for y in [-maxR, imgY); fine_pixel_coor yields x < max(imgX, maxR + 1)
  // and -maxR <= y < imgY.
  extern __shared__ float2 s_tab[];
  const int exw = max(v.imgX, v.maxR + 1), eyw = v.imgY + v.maxR;
  float2* s_ex = s_tab;
  float2* s_ey = s_tab + NT * exw;
  for (int base = 0; base < ntrans; base += NT) {  // passes of NT translations
    const int nt = min(NT, ntrans - base);
    float ftx[NT], fty[NT], acc[NT];
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      ftx[i] = i < nt ? tx[t0 + base + i] : 0.f;
      fty[i] = i < nt ? ty[t0 + base + i] : 0.f;
      acc[i] = 0.f;
    }
    if (TABLES) {
      for (int e2 = threadIdx.x; e2 < NT * (exw + eyw); e2 += kFineThreads) {
        float sn = 0.f, cs = 1.f;
        if (e2 < NT * exw) {
          const int i = e2 / exw, x = e2 - i * exw;
          if (i < nt) sincosf(__fmul_rn((float)x, tx[t0 + base + i]), &sn, &cs);
          s_ex[e2] = make_float2(cs, sn);
        } else {
          const int j = e2 - NT * exw, i = j / eyw, y = j - i * eyw - v.maxR;
          if (i < nt) sincosf(__fmul_rn((float)y, ty[t0 + base + i]), &sn, &cs);
          s_ey[j] = make_float2(cs, sn);
        }
      }
      __syncthreads();
    }
    double nrm = 0.0;  // this thread's sum w(|A|^2 + |X|^2) (tables) or sum corr |A|^2 (CC)
    for (int pixel = threadIdx.x; pixel < image_size; pixel += kFineThreads) {
      int x, y;
      fine_pixel_coor(pixel, v.imgX, v.imgY, v.maxR, x, y);
      const float2 a = project_pixel(v, (float)x, (float)y, e);
      const float xr = re[pixel], xi = im[pixel];
      const float w = CC ? corr[pixel] : 0.5f * corr[pixel];
      if (CC) {  // the CC denominator: sum corr |A|^2
        const double ad = a.x, bd = a.y;
        nrm = fma((double)w, fma(ad, ad, bd * bd), nrm);
      }
      if (TABLES) {
        const double ad = a.x, bd = a.y, xd = xr, yd = xi;
        if (!CC) nrm = fma((double)w, fma(ad, ad, fma(bd, bd, fma(xd, xd, yd * yd))), nrm);
        const float qr = __fmul_rn(w, __fmaf_rn(a.x, xr, __fmul_rn(a.y, xi)));   // w Re(conj(A) X)
        const float qi = __fmul_rn(w, __fmaf_rn(a.x, xi, -__fmul_rn(a.y, xr)));  // w Im(conj(A) X)
        const float2* pex = s_ex + x;
        const float2* pey = s_ey + y + v.maxR;
#pragma unroll
        for (int i = 0; i < NT; ++i) {
          if (i < nt) {
            const float2 ex = pex[i * exw], ey = pey[i * eyw];
            const float ur = __fmaf_rn(qr, ex.x, -__fmul_rn(qi, ex.y));
            const float ui = __fmaf_rn(qr, ex.y, __fmul_rn(qi, ex.x));
            acc[i] = __fmaf_rn(ur, ey.x, __fmaf_rn(-ui, ey.y, acc[i]));
          }
        }
      } else {
#pragma unroll
        for (int i = 0; i < NT; ++i) {
          if (i < nt) {
            float s, c;
            sincosf(__fmaf_rn((float)x, ftx[i], __fmul_rn((float)y, fty[i])), &s, &c);
            if (CC) {  // corr Re(conj(A) S), S = X e^{i(x tx + y ty)}
              const float sr = __fmaf_rn(c, xr, -__fmul_rn(s, xi));
              const float si = __fmaf_rn(c, xi, __fmul_rn(s, xr));
              acc[i] = __fmaf_rn(__fmaf_rn(a.x, sr, __fmul_rn(a.y, si)), w, acc[i]);
              continue;
            }
            const float dr = a.x - __fmaf_rn(c, xr, -__fmul_rn(s, xi));
            const float di = a.y - __fmaf_rn(c, xi, __fmul_rn(s, xr));
            acc[i] = __fmaf_rn(__fmaf_rn(dr, dr, __fmul_rn(di, di)), w, acc[i]);
          }
        }
      }
    }
    // fixed-order reduction: shuffle tree inside each warp, then warps in order
    if (TABLES || CC) {
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        double vsum = (double)acc[i];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) vsum += __shfl_xor_sync(0xffffffffu, vsum, off);
        if ((threadIdx.x & 31) == 0) s_cross[threadIdx.x >> 5][i] = vsum;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, off);
      if ((threadIdx.x & 31) == 0) s_norm[threadIdx.x >> 5] = nrm;
    } else {
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        float vsum = acc[i];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) vsum += __shfl_xor_sync(0xffffffffu, vsum, off);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5][i] = vsum;
      }
    }
    __syncthreads();
    if (threadIdx.x < nt) {
      if (TABLES || CC) {
        double cr = 0.0, nt2 = 0.0;
#pragma unroll
        for (int w = 0; w < kFineThreads / 32; ++w) {
          cr += s_cross[w][threadIdx.x];
          nt2 += s_norm[w];
        }
        diff2s[jb + base + threadIdx.x] = CC ? (float)(-cr / sqrt(nt2)) : (float)(fma(-2.0, cr, nt2) + (double)sum_init);
      } else {
        float tot = 0.f;
#pragma unroll
        for (int w = 0; w < kFineThreads / 32; ++w) tot += s_part[w][threadIdx.x];
        diff2s[jb + base + threadIdx.x] = tot + sum_init;
      }
    }
    __syncthreads();
  }
}

}  // namespace b200d2

namespace {

template <bool CC>
int launch_fine(const b200d2_view* view, const float* d_eulers, const float* d_real, const float* d_imag,
                const float* d_trans_x, const float* d_trans_y, const float* d_corr, float* d_diff2s,
                size_t image_size, float sum_init, size_t todo_blocks, const uint64_t* d_rot_idx,
                const uint64_t* d_trans_idx, const uint64_t* d_job_idx, const uint64_t* d_job_num, void* stream) {
  using namespace b200d2;
  if (!view) return B200D2_ERR_INVALID;
  if (todo_blocks == 0 || image_size == 0) return B200D2_OK;
  if (!d_eulers || !d_real || !d_imag || !d_trans_x || !d_trans_y || !d_corr || !d_diff2s || !d_rot_idx ||
      !d_trans_idx || !d_job_idx || !d_job_num)
    return B200D2_ERR_INVALID;
  if (view->mdlZ == 0) return B200D2_ERR_UNSUPPORTED;  // 2D references are outside the ported branch
  if ((long long)view->imgX * view->imgY < (long long)image_size || image_size > 0x7fffffffull)
    return B200D2_ERR_INVALID;
  if (view->interp == B200D2_INTERP_TEXTURE && (!view->tex_re || !view->tex_im)) return B200D2_ERR_INVALID;
  if (view->interp == B200D2_INTERP_LINEAR && (!view->lin_re || !view->lin_im)) return B200D2_ERR_INVALID;
  if (todo_blocks > 0x7fffffffull) return B200D2_ERR_UNSUPPORTED;
  const size_t exw = (size_t)std::max(view->imgX, view->maxR + 1);
  const size_t tab_bytes = sizeof(float2) * kFineMaxTrans * (exw + view->imgY + view->maxR);
  if (view->maxR >= 0 && view->imgX > 0 && view->imgY > 0 && tab_bytes <= kFineTableBytes) {
    static bool attr = false;  // the opt-in above 48 KB of dynamic shared memory
    if (!attr) {
      B200D2_CUDA_TRY(cudaFuncSetAttribute(diff2_fine_kernel<kFineMaxTrans, true, CC>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFineTableBytes));
      attr = true;
    }
    diff2_fine_kernel<kFineMaxTrans, true, CC><<<(unsigned)todo_blocks, kFineThreads, tab_bytes,
                                                 (cudaStream_t)stream>>>(
        *view, d_eulers, d_real, d_imag, d_trans_x, d_trans_y, d_corr, d_diff2s, (int)image_size, sum_init,
        d_rot_idx, d_trans_idx, d_job_idx, d_job_num);
  } else {
    diff2_fine_kernel<kFineMaxTrans, false, CC><<<(unsigned)todo_blocks, kFineThreads, 0, (cudaStream_t)stream>>>(
        *view, d_eulers, d_real, d_imag, d_trans_x, d_trans_y, d_corr, d_diff2s, (int)image_size, sum_init,
        d_rot_idx, d_trans_idx, d_job_idx, d_job_num);
  }
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

}  // namespace

extern "C" int b200d2_diff2_fine(const b200d2_view* view, const float* d_eulers, const float* d_real,
                                 const float* d_imag, const float* d_trans_x, const float* d_trans_y,
                                 const float* d_corr, float* d_diff2s, size_t image_size, float sum_init,
                                 size_t todo_blocks, const uint64_t* d_rot_idx, const uint64_t* d_trans_idx,
                                 const uint64_t* d_job_idx, const uint64_t* d_job_num, void* stream) {
  return launch_fine<false>(view, d_eulers, d_real, d_imag, d_trans_x, d_trans_y, d_corr, d_diff2s, image_size,
                            sum_init, todo_blocks, d_rot_idx, d_trans_idx, d_job_idx, d_job_num, stream);
}

extern "C" int b200d2_diff2_fine_cc(const b200d2_view* view, const float* d_eulers, const float* d_real,
                                    const float* d_imag, const float* d_trans_x, const float* d_trans_y,
                                    const float* d_corr, float* d_diff2s, size_t image_size, size_t todo_blocks,
                                    const uint64_t* d_rot_idx, const uint64_t* d_trans_idx,
                                    const uint64_t* d_job_idx, const uint64_t* d_job_num, void* stream) {
  return launch_fine<true>(view, d_eulers, d_real, d_imag, d_trans_x, d_trans_y, d_corr, d_diff2s, image_size,
                           0.f, todo_blocks, d_rot_idx, d_trans_idx, d_job_idx, d_job_num, stream);
}
