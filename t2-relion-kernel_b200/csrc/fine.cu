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

// Table path with the phase factored by rows.  With e^{i(x tx + y ty)} =
// e^{i x tx} e^{i y ty},
//   sum_px Re(q e^{i x tx} e^{i y ty}) = sum_x Re(e^{i x tx} R(x)),  R(x) = sum_y q(x, y) e^{i y ty}.
// A thread owns one image column and a contiguous range of its rows.  Phase
// 1: it projects its pixels once per job (four in flight) and keeps
// q = w conj(A) X in shared memory, with the per-pixel FP64 norms of
// diff2_fine_kernel.  Phase 2: it accumulates R for the job's translations,
// one complex multiply-add per (pixel, translation), the row's phases of two
// translations in one 16-byte shared-memory load (the same address for every
// lane of a row); e^{i x tx} is applied once at the end.  Rows that the fine
// mapping sends to x = maxR (between maxR and imgY - maxR) lie outside the
// projector radius, so their q is zero; a nonzero q there enters R(col) as
// q e^{i x' tx} conj(e^{i col tx}) e^{i y ty} (x' = maxR).  The 16 partial
// cross sums of a warp are reduced by halving exchanges (16 shuffles of
// doubles instead of 80) in a fixed order, then warps in order.  The y table
// covers the rows' y after the mapping, [-maxR, max(maxR, imgY - maxR - 1)].
constexpr int kFineColsMaxThreads = 288;
__host__ __device__ inline int fine_cols_eyw(int imgY, int maxR) { return maxR + max(maxR, imgY - maxR - 1) + 1; }
constexpr size_t kFineColsSmem = 160 * 1024;  // tables + q, per CTA

template <int NT, bool CC>
__global__ void __launch_bounds__(kFineColsMaxThreads, 3) diff2_fine_cols_kernel(
    b200d2_view v, const float* __restrict__ eulers, const float* __restrict__ re, const float* __restrict__ im,
    const float* __restrict__ tx, const float* __restrict__ ty, const float* __restrict__ corr,
    float* __restrict__ diff2s, int image_size, float sum_init, int groups, const uint64_t* __restrict__ rot_idx,
    const uint64_t* __restrict__ trans_idx, const uint64_t* __restrict__ job_idx,
    const uint64_t* __restrict__ job_num) {
  static_assert(NT == 16, "the warp reduction below is written for 16 translations");
  constexpr int kWarpsMax = kFineColsMaxThreads / 32;
  const uint64_t jb = job_idx[blockIdx.x];
  const int ntrans = (int)job_num[blockIdx.x];
  const uint64_t o = rot_idx[jb];
  const uint64_t t0 = trans_idx[jb];
  const float* eo = eulers + o * 9;
  const float e[6] = {eo[0], eo[1], eo[3], eo[4], eo[6], eo[7]};
  __shared__ double s_cross[kWarpsMax][NT], s_norm[kWarpsMax];
  extern __shared__ __align__(16) float2 s_tab[];
  const int exw = max(v.imgX, v.maxR + 1), eyw = fine_cols_eyw(v.imgY, v.maxR);
  float2* s_ex = s_tab;             // [NT][exw], x fastest
  float2* s_ey = s_tab + NT * exw;  // [eyw][NT], translation fastest, row y + maxR
  float2* s_q = s_ey + NT * eyw;    // [image_size]
  const int nthr = blockDim.x, nwarps = nthr >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = threadIdx.x % v.imgX, grp = threadIdx.x / v.imgX;
  const bool active = grp < groups;
  const int y0 = active ? (int)((long long)grp * v.imgY / groups) : 0;
  const int y1 = active ? (int)((long long)(grp + 1) * v.imgY / groups) : 0;
  // phase 1 (once per job): q of this thread's pixels and its norm
  double nrm = 0.0;
  constexpr int kQ = 4;
  for (int yb = y0; yb < y1; yb += kQ) {
    int pix[kQ];
    float2 a[kQ];
#pragma unroll
    for (int u = 0; u < kQ; ++u) {
      const int ys = yb + u;
      pix[u] = ys < y1 ? ys * v.imgX + col : image_size;
      a[u] = make_float2(0.f, 0.f);
      if (pix[u] < image_size) {
        int x = col, y = ys;
        if (y > v.maxR) {  // the fine kernel's mapping (fine_pixel_coor)
          if (y >= v.imgY - v.maxR)
            y -= v.imgY;
          else
            x = v.maxR;
        }
        a[u] = project_pixel(v, (float)x, (float)y, e);
      }
    }
#pragma unroll
    for (int u = 0; u < kQ; ++u) {
      if (pix[u] >= image_size) continue;
      const float xr = re[pix[u]], xi = im[pix[u]];
      const float w = CC ? corr[pix[u]] : 0.5f * corr[pix[u]];
      const double ad = a[u].x, bd = a[u].y;
      if (CC) {
        nrm = fma((double)w, fma(ad, ad, bd * bd), nrm);
      } else {
        const double xd = xr, yd = xi;
        nrm = fma((double)w, fma(ad, ad, fma(bd, bd, fma(xd, xd, yd * yd))), nrm);
      }
      s_q[pix[u]] = make_float2(__fmul_rn(w, __fmaf_rn(a[u].x, xr, __fmul_rn(a[u].y, xi))),    // w Re(conj(A) X)
                                __fmul_rn(w, __fmaf_rn(a[u].x, xi, -__fmul_rn(a[u].y, xr))));  // w Im(conj(A) X)
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, off);
  if (lane == 0) s_norm[warp] = nrm;
  for (int base = 0; base < ntrans; base += NT) {  // passes of NT translations
    const int nt = min(NT, ntrans - base);
    for (int e2 = threadIdx.x; e2 < NT * (exw + eyw); e2 += nthr) {
      float sn = 0.f, cs = 1.f;
      if (e2 < NT * exw) {
        const int i = e2 / exw, x = e2 - i * exw;
        if (i < nt) sincosf(__fmul_rn((float)x, tx[t0 + base + i]), &sn, &cs);
      } else {
        const int j = e2 - NT * exw, yy = j / NT, i = j - yy * NT;
        if (i < nt) sincosf(__fmul_rn((float)(yy - v.maxR), ty[t0 + base + i]), &sn, &cs);
      }
      s_tab[e2] = make_float2(cs, sn);
    }
    __syncthreads();  // tables (and, on the first pass, q and the norms) ready
    // phase 2: R for this thread's column and rows
    float rr[NT], ri[NT];
#pragma unroll
    for (int i = 0; i < NT; ++i) rr[i] = ri[i] = 0.f;
    for (int ys = y0; ys < y1; ++ys) {
      const int pixel = ys * v.imgX + col;
      if (pixel >= image_size) break;  // later rows of this column lie further on
      const float2 q = s_q[pixel];
      int x = col, y = ys;
      if (y > v.maxR) {  // the fine kernel's mapping (fine_pixel_coor)
        if (y >= v.imgY - v.maxR)
          y -= v.imgY;
        else
          x = v.maxR;
      }
      if (x == col) {
        const float4* pey = reinterpret_cast<const float4*>(s_ey + (y + v.maxR) * NT);
#pragma unroll
        for (int k = 0; k < NT / 2; ++k) {
          const float4 f = pey[k];  // (cos, sin) of translations 2k and 2k + 1
          rr[2 * k] = __fmaf_rn(q.x, f.x, __fmaf_rn(-q.y, f.y, rr[2 * k]));
          ri[2 * k] = __fmaf_rn(q.x, f.y, __fmaf_rn(q.y, f.x, ri[2 * k]));
          rr[2 * k + 1] = __fmaf_rn(q.x, f.z, __fmaf_rn(-q.y, f.w, rr[2 * k + 1]));
          ri[2 * k + 1] = __fmaf_rn(q.x, f.w, __fmaf_rn(q.y, f.z, ri[2 * k + 1]));
        }
      } else if (q.x != 0.f || q.y != 0.f) {  // a remapped row with a nonzero projection
        const float2* pey = s_ey + (y + v.maxR) * NT;
#pragma unroll
        for (int i = 0; i < NT; ++i) {
          const float2 ex = s_ex[i * exw + x], cx = s_ex[i * exw + col], ey = pey[i];
          // d = e^{i x' tx} conj(e^{i col tx}) e^{i y ty}
          const float dr0 = __fmaf_rn(ex.x, cx.x, __fmul_rn(ex.y, cx.y));
          const float di0 = __fmaf_rn(ex.y, cx.x, -__fmul_rn(ex.x, cx.y));
          const float dr = __fmaf_rn(dr0, ey.x, -__fmul_rn(di0, ey.y));
          const float di = __fmaf_rn(dr0, ey.y, __fmul_rn(di0, ey.x));
          rr[i] = __fmaf_rn(q.x, dr, __fmaf_rn(-q.y, di, rr[i]));
          ri[i] = __fmaf_rn(q.x, di, __fmaf_rn(q.y, dr, ri[i]));
        }
      }
    }
    // this thread's cross sums Re(e^{i col tx} R), then the warp's 16 sums by
    // halving exchanges: after the exchanges at distance 16, 8, 4 and 2, lane
    // l holds translation 8 b4 + 4 b3 + 2 b2 + b1 (b_k: bit k of l) summed over
    // its 16-lane group; distance 1 adds the two groups.
    double c[NT];
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const float2 f = s_ex[i * exw + col];
      c[i] = active ? (double)__fmaf_rn(f.x, rr[i], -__fmul_rn(f.y, ri[i])) : 0.0;
    }
#pragma unroll
    for (int h = NT / 2; h >= 1; h >>= 1) {
      const int dist = 2 * h;  // 16, 8, 4, 2
      const bool up = lane & dist;
#pragma unroll
      for (int k = 0; k < h; ++k) {
        const double send = up ? c[k] : c[k + h];
        const double keep = up ? c[k + h] : c[k];
        c[k] = keep + __shfl_xor_sync(0xffffffffu, send, dist);
      }
    }
    const double tot = c[0] + __shfl_xor_sync(0xffffffffu, c[0], 1);
    const int my_t = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    if ((lane & 1) == 0) s_cross[warp][my_t] = tot;
    __syncthreads();
    if (threadIdx.x < nt) {
      double cr = 0.0, nt2 = 0.0;
      for (int w = 0; w < nwarps; ++w) {
        cr += s_cross[w][threadIdx.x];
        nt2 += s_norm[w];
      }
      diff2s[jb + base + threadIdx.x] =
          CC ? (float)(-cr / sqrt(nt2)) : (float)(fma(-2.0, cr, nt2) + (double)sum_init);
    }
    __syncthreads();  // s_cross and the tables are reused by the next pass
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
  const size_t cols_bytes =  // tables + q
      sizeof(float2) * (kFineMaxTrans * (exw + (size_t)fine_cols_eyw(view->imgY, view->maxR)) + image_size);
  if (view->maxR >= 0 && view->imgX > 0 && view->imgY > 0 && cols_bytes <= kFineColsSmem &&
      view->imgX <= kFineColsMaxThreads) {
    // one thread per (column, row group), about 256 threads, whole warps
    const int groups = std::max(1, std::min(view->imgY, std::min((256 + view->imgX / 2) / view->imgX,
                                                                  kFineColsMaxThreads / view->imgX)));
    const int threads = (view->imgX * groups + 31) / 32 * 32;
    static std::atomic<unsigned long long> opted{0};  // above 48 KB of dynamic shared memory
    B200D2_CUDA_TRY(smem_opt_in(diff2_fine_cols_kernel<kFineMaxTrans, CC>, (int)kFineColsSmem, opted));
    diff2_fine_cols_kernel<kFineMaxTrans, CC><<<(unsigned)todo_blocks, threads, cols_bytes, (cudaStream_t)stream>>>(
        *view, d_eulers, d_real, d_imag, d_trans_x, d_trans_y, d_corr, d_diff2s, (int)image_size, sum_init, groups,
        d_rot_idx, d_trans_idx, d_job_idx, d_job_num);
  } else if (view->maxR >= 0 && view->imgX > 0 && view->imgY > 0 && tab_bytes <= kFineTableBytes) {
    static std::atomic<unsigned long long> opted{0};  // above 48 KB of dynamic shared memory
    B200D2_CUDA_TRY(smem_opt_in(diff2_fine_kernel<kFineMaxTrans, true, CC>, (int)kFineTableBytes, opted));
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
