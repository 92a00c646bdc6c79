// diff2_direct.cu -- plain CUDA-core coarse diff2 (FP32 drop-in, FP64 oracle).
//
// Semantics of cuda_kernel_diff2_coarse (src/diff2.cuh:369-537) and its FP64
// twin (src/diff2.cuh:205-365): for every orientation o and translation t
//   diff2s[o*T + t] += sum_{px < N_img} ((A_o - S_t)_re^2 + (A_o - S_t)_im^2) * corr/2
// with A_o the projection (project3Dmodel) and S_t the phase-shifted image
// (translatePixel).  The per-term arithmetic is the reference's: difference,
// squared magnitude, times corr/2, accumulated in the working precision.
//
// B200 design (not the reference's loop structure):
//  * one CTA owns a BT x BO (translation x orientation) output tile of one
//    particle and walks the whole image, so each output is written once (no
//    atomics, deterministic order) and accumulates onto the caller's value;
//  * pixels are streamed in chunks of 256; a ballot compaction keeps only the
//    pixels some orientation can see (the rest contribute |S|^2 corr/2 =
//    |X|^2 corr/2 to every (o, t), added once per CTA);
//  * per 16-pixel sub-chunk the CTA stages the shifted image S[k][t] (one
//    sincos per (t, k)) and the projections A[k][o] (one texture pair per
//    (o, k)) in shared memory; every thread then keeps a TT x TO register tile
//    whose inner step is 5 FP32 instructions per (o, t, pixel);
//  * thread (tq, oq) owns translations tq + 16 i and orientations oq + 16 j,
//    so a warp reads S conflict-free and A as a broadcast.
//
// The CC form (cuda_kernel_diff2_CC_coarse, src/diff2.cuh:691-809) runs the
// same tiles with corr as the weight: the register tile accumulates
// sum corr Re(conj(A) S) and each thread keeps sum corr |A|^2 of its
// orientations; the output is -cross / sqrt(norm), written (or added with
// accumulate).  Pixels outside the projector radius have A = 0 and are skipped.
#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"

namespace b200d2 {

struct DirectArgs {
  b200d2_view view;
  const float* eulers;
  const float* trans_x;
  const float* trans_y;
  const float* re;
  const float* im;
  const float* corr;
  void* diff2;
  long long img_stride;  // elements between consecutive particles' images
  long long out_stride;  // elements between consecutive particles' outputs
  int O, T, N_img;
  int o_tiles;
  int filter_img;
  int cc;          // 1: cross-correlation score
  int accumulate;  // CC: add onto the output instead of writing it
};

template <typename R>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

template <typename R>
__device__ __forceinline__ typename Vec2<R>::type shift_pixel(float fx, float fy,
                                                             float tx, float ty,
                                                             float re, float im);

template <>
__device__ __forceinline__ float2 shift_pixel<float>(float fx, float fy,
                                                     float tx, float ty,
                                                     float re, float im) {
  float s, c;
  sincosf(__fmaf_rn(fx, tx, __fmul_rn(fy, ty)), &s, &c);
  return make_float2(__fmaf_rn(c, re, -__fmul_rn(s, im)),
                     __fmaf_rn(c, im, __fmul_rn(s, re)));
}

template <>
__device__ __forceinline__ double2 shift_pixel<double>(float fx, float fy,
                                                       float tx, float ty,
                                                       float re, float im) {
  double s, c;
  sincos((double)fx * (double)tx + (double)fy * (double)ty, &s, &c);
  return make_double2(c * (double)re - s * (double)im,
                      c * (double)im + s * (double)re);
}

template <typename R, int TT, int TO, int KC, bool CC>
__global__ void __launch_bounds__(256) diff2_direct_kernel(const DirectArgs a) {
  using R2 = typename Vec2<R>::type;
  constexpr int BT = 16 * TT, BO = 16 * TO, NT = 256, RAW = 256;
  __shared__ float s_eul[BO][6];
  __shared__ float s_tx[BT], s_ty[BT];
  __shared__ short2 s_xy[RAW];
  __shared__ float s_re[RAW], s_im[RAW], s_w[RAW];
  __shared__ R2 s_S[KC][BT];
  __shared__ R2 s_A[KC][BO];
  __shared__ R s_wk[KC];
  __shared__ int s_cnt[8];
  __shared__ R s_red[8];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long p = blockIdx.z;
  const int o0 = (blockIdx.x % a.o_tiles) * BO;
  const int t0 = (blockIdx.x / a.o_tiles) * BT;
  const b200d2_view& v = a.view;
  const float* __restrict__ g_re = a.re + p * a.img_stride;
  const float* __restrict__ g_im = a.im + p * a.img_stride;
  const float* __restrict__ g_corr = a.corr + p * a.img_stride;

  for (int i = tid; i < BO * 6; i += NT) {
    const int o = o0 + i / 6, c = i % 6;
    const int src = (c >> 1) * 3 + (c & 1);  // e0 e1 e3 e4 e6 e7
    s_eul[i / 6][c] = o < a.O ? a.eulers[(size_t)o * 9 + src] : 0.f;
  }
  for (int i = tid; i < BT; i += NT) {
    const int t = t0 + i;
    s_tx[i] = t < a.T ? a.trans_x[t] : 0.f;
    s_ty[i] = t < a.T ? a.trans_y[t] : 0.f;
  }

  const int tq = tid & 15, oq = tid >> 4;
  R acc[TT][TO];
  R nrm[TO];
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TO; ++j) acc[i][j] = R(0);
#pragma unroll
  for (int j = 0; j < TO; ++j) nrm[j] = R(0);
  R out_part = R(0);

  for (int base = 0; base < a.N_img; base += RAW) {
    __syncthreads();
    const int i = base + tid;
    bool in = false;
    int x = 0, y = 0;
    float re = 0.f, im = 0.f, w = 0.f;
    if (i < a.N_img) {
      pixel_coor(i, v.imgX, v.imgY, v.maxR, x, y);
      re = g_re[i];
      im = g_im[i];
      w = CC ? g_corr[i] : g_corr[i] / 2;
      in = pixel_maybe_inside(x, y, v.padding_factor, v.maxR2_padded);
      if (a.filter_img) {
        // reference filter test (src/diff2.cuh:339-345), in double
        double r2 = (double)(x * x + y * y) * v.padding_factor * v.padding_factor;
        if (r2 > (double)v.maxR2_padded) re = im = 0.f;
      }
      if (!CC && !in) {
        const R rr = (R)re, ri = (R)im;
        out_part += (rr * rr + ri * ri) * (R)w;
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    if (lane == 0) s_cnt[warp] = __popc(bal);
    __syncthreads();
    int off = 0, total = 0;
#pragma unroll
    for (int w2 = 0; w2 < 8; ++w2) {
      const int c = s_cnt[w2];
      off += (w2 < warp) ? c : 0;
      total += c;
    }
    if (in) {
      const int slot = off + __popc(bal & ((1u << lane) - 1u));
      s_xy[slot] = make_short2((short)x, (short)y);
      s_re[slot] = re;
      s_im[slot] = im;
      s_w[slot] = w;
    }
    __syncthreads();

    for (int k0 = 0; k0 < total; k0 += KC) {
      for (int e = tid; e < KC * BT; e += NT) {
        const int k = e / BT, t = e % BT;
        R2 sv;
        sv.x = R(0);
        sv.y = R(0);
        if (k0 + k < total) {
          const short2 xy = s_xy[k0 + k];
          sv = shift_pixel<R>((float)xy.x, (float)xy.y, s_tx[t], s_ty[t],
                              s_re[k0 + k], s_im[k0 + k]);
        }
        s_S[k][t] = sv;
      }
      for (int e = tid; e < KC * BO; e += NT) {
        const int k = e / BO, o = e % BO;
        float2 pr = make_float2(0.f, 0.f);
        if (k0 + k < total && o0 + o < a.O) {
          const short2 xy = s_xy[k0 + k];
          pr = project_pixel(v, (float)xy.x, (float)xy.y, s_eul[o]);
        }
        R2 av;
        av.x = (R)pr.x;
        av.y = (R)pr.y;
        s_A[k][o] = av;
      }
      if (tid < KC) s_wk[tid] = (k0 + tid < total) ? (R)s_w[k0 + tid] : R(0);
      __syncthreads();
#pragma unroll 4
      for (int k = 0; k < KC; ++k) {
        const R w = s_wk[k];
        R2 sv[TT], av[TO];
#pragma unroll
        for (int ii = 0; ii < TT; ++ii) sv[ii] = s_S[k][tq + 16 * ii];
#pragma unroll
        for (int j = 0; j < TO; ++j) av[j] = s_A[k][oq + 16 * j];
        if (CC) {
#pragma unroll
          for (int j = 0; j < TO; ++j) nrm[j] = fma(fma(av[j].x, av[j].x, av[j].y * av[j].y), w, nrm[j]);
#pragma unroll
          for (int ii = 0; ii < TT; ++ii)
#pragma unroll
            for (int j = 0; j < TO; ++j)
              acc[ii][j] = fma(fma(av[j].x, sv[ii].x, av[j].y * sv[ii].y), w, acc[ii][j]);
        } else {
#pragma unroll
          for (int ii = 0; ii < TT; ++ii)
#pragma unroll
            for (int j = 0; j < TO; ++j) {
              const R dr = av[j].x - sv[ii].x;
              const R di = av[j].y - sv[ii].y;
              acc[ii][j] = fma(fma(dr, dr, di * di), w, acc[ii][j]);
            }
        }
      }
      __syncthreads();
    }
  }

  // block-reduce the out-of-radius constant
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) out_part += __shfl_xor_sync(0xffffffffu, out_part, o);
  if (lane == 0) s_red[warp] = out_part;
  __syncthreads();
  R out_total = R(0);
#pragma unroll
  for (int w2 = 0; w2 < 8; ++w2) out_total += s_red[w2];

  R* __restrict__ g_out = reinterpret_cast<R*>(a.diff2) + p * a.out_stride;
#pragma unroll
  for (int ii = 0; ii < TT; ++ii) {
    const int t = t0 + tq + 16 * ii;
    if (t >= a.T) continue;
#pragma unroll
    for (int j = 0; j < TO; ++j) {
      const int o = o0 + oq + 16 * j;
      if (o < a.O) {
        R* dst = g_out + (size_t)o * a.T + t;
        if (CC) {
          const R cc = -(acc[ii][j] / sqrt(nrm[j]));
          *dst = a.accumulate ? *dst + cc : cc;
        } else {
          *dst = *dst + (acc[ii][j] + out_total);
        }
      }
    }
  }
}

template <typename R, int TT, int TO, bool CC>
static int launch_tt_to(const DirectArgs& a0, int P, cudaStream_t s) {
  constexpr int KC = std::is_same<R, double>::value ? 8 : 16;
  DirectArgs a = a0;
  a.o_tiles = (a.O + 16 * TO - 1) / (16 * TO);
  const int t_tiles = (a.T + 16 * TT - 1) / (16 * TT);
  const long long nx = (long long)a.o_tiles * t_tiles;
  if (nx > 0x7fffffffLL || P > 65535) return B200D2_ERR_UNSUPPORTED;
  dim3 grid((unsigned)nx, 1, (unsigned)P);
  diff2_direct_kernel<R, TT, TO, KC, CC><<<grid, 256, 0, s>>>(a);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

template <typename R, int TT, bool CC>
static int launch_tt(const DirectArgs& a, int P, int to, cudaStream_t s) {
  if (to >= 8) return launch_tt_to<R, TT, (std::is_same<R, double>::value ? 4 : 8), CC>(a, P, s);
  if (to >= 4) return launch_tt_to<R, TT, 4, CC>(a, P, s);
  return launch_tt_to<R, TT, 2, CC>(a, P, s);
}

// Tile choice: BT = 16*TT just covers T (up to 128, larger T uses several
// translation tiles); BO = 16*TO is the largest of 128/64/32 that still gives
// at least two CTAs per SM.
template <typename R>
static int launch_direct(const DirectArgs& a, int P, cudaStream_t s) {
  if (a.O <= 0 || a.T <= 0 || a.N_img <= 0 || P <= 0) return B200D2_OK;
  int tt = a.T <= 16 ? 1 : a.T <= 32 ? 2 : a.T <= 64 ? 4 : 8;
  const int t_tiles = (a.T + 16 * tt - 1) / (16 * tt);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int to = 8;
  while (to > 2 && (long long)P * t_tiles * ((a.O + 16 * to - 1) / (16 * to)) < 2LL * sms)
    to >>= 1;
  if (a.cc) {
    switch (tt) {
      case 1: return launch_tt<R, 1, true>(a, P, to, s);
      case 2: return launch_tt<R, 2, true>(a, P, to, s);
      case 4: return launch_tt<R, 4, true>(a, P, to, s);
      default: return launch_tt<R, 8, true>(a, P, to, s);
    }
  }
  switch (tt) {
    case 1: return launch_tt<R, 1, false>(a, P, to, s);
    case 2: return launch_tt<R, 2, false>(a, P, to, s);
    case 4: return launch_tt<R, 4, false>(a, P, to, s);
    default: return launch_tt<R, 8, false>(a, P, to, s);
  }
}

static int check_common(const b200d2_view* view, const void* tx, const void* ty,
                        const void* corr, const void* re, const void* im,
                        const void* eul, const void* out, size_t O, size_t T,
                        size_t N_img) {
  if (!view || !tx || !ty || !corr || !re || !im || !eul || !out)
    return B200D2_ERR_INVALID;
  if (O > 0x7fffffff || T > 0x7fffffff || N_img > 0x7fffffff) return B200D2_ERR_INVALID;
  if ((size_t)view->imgX * (size_t)view->imgY < N_img) return B200D2_ERR_INVALID;
  if (view->mdlZ == 0) return B200D2_ERR_UNSUPPORTED;
  if (view->interp == B200D2_INTERP_TEXTURE && (!view->tex_re || !view->tex_im))
    return B200D2_ERR_INVALID;
  if (view->interp == B200D2_INTERP_LINEAR && (!view->lin_re || !view->lin_im))
    return B200D2_ERR_INVALID;
  if (view->imgX > 32767 || view->imgY > 32767) return B200D2_ERR_UNSUPPORTED;
  return B200D2_OK;
}

// Batched entry used by the library's own batch API and benchmarks: P
// particles sharing eulers and translations, images and outputs strided.
int direct_batch(const b200d2_view& view, const float* eulers, const float* tx,
                 const float* ty, const float* re, const float* im,
                 const float* corr, long long img_stride, void* out,
                 long long out_stride, int O, int T, int N_img, int P,
                 bool fp64, int filter_img, cudaStream_t s, int cc, int accumulate) {
  DirectArgs a;
  a.view = view;
  a.eulers = eulers;
  a.trans_x = tx;
  a.trans_y = ty;
  a.re = re;
  a.im = im;
  a.corr = corr;
  a.diff2 = out;
  a.img_stride = img_stride;
  a.out_stride = out_stride;
  a.O = O;
  a.T = T;
  a.N_img = N_img;
  a.o_tiles = 1;
  a.filter_img = filter_img;
  a.cc = cc;
  a.accumulate = accumulate;
  return fp64 ? launch_direct<double>(a, P, s) : launch_direct<float>(a, P, s);
}

}  // namespace b200d2

namespace b200d2 {
int single_particle_tc(const b200d2_view& v, const float* tx, const float* ty, const float* corr, const float* re,
                       const float* im, const float* eulers, float* diff2s, int O, int T, int N_img, int precision,
                       cudaStream_t s);
}  // namespace b200d2

extern "C" int b200d2_diff2_coarse(const b200d2_view* view,
                                   const float* d_trans_x,
                                   const float* d_trans_y, const float* d_corr,
                                   const float* d_real, const float* d_imag,
                                   const float* d_eulers, float* d_diff2s,
                                   size_t O, size_t T, size_t N_img,
                                   void* stream, int precision) {
  b200d2::NvtxRange range("b200d2_diff2_coarse");
  int st = b200d2::check_common(view, d_trans_x, d_trans_y, d_corr, d_real,
                                d_imag, d_eulers, d_diff2s, O, T, N_img);
  if (st != B200D2_OK) return st;
  if (b200d2::is_tc_precision(precision)) {
    if (O > 0x7fffffff || T > 0x7fffffff || N_img > 0x7fffffff) return B200D2_ERR_UNSUPPORTED;
    return b200d2::single_particle_tc(*view, d_trans_x, d_trans_y, d_corr, d_real, d_imag, d_eulers, d_diff2s,
                                      (int)O, (int)T, (int)N_img, precision, (cudaStream_t)stream);
  }
  if (precision != B200D2_PREC_FP32) return B200D2_ERR_UNSUPPORTED;
  return b200d2::direct_batch(*view, d_eulers, d_trans_x, d_trans_y, d_real,
                              d_imag, d_corr, 0, d_diff2s, 0, (int)O, (int)T,
                              (int)N_img, 1, false, 0, (cudaStream_t)stream, 0, 1);
}

extern "C" int b200d2_diff2_coarse_f64(const b200d2_view* view,
                                       const float* d_trans_x,
                                       const float* d_trans_y,
                                       const float* d_corr,
                                       const float* d_real,
                                       const float* d_imag,
                                       const float* d_eulers, double* d_diff2s,
                                       size_t O, size_t T, size_t N_img,
                                       int filter_img, void* stream) {
  int st = b200d2::check_common(view, d_trans_x, d_trans_y, d_corr, d_real,
                                d_imag, d_eulers, d_diff2s, O, T, N_img);
  if (st != B200D2_OK) return st;
  return b200d2::direct_batch(*view, d_eulers, d_trans_x, d_trans_y, d_real,
                              d_imag, d_corr, 0, d_diff2s, 0, (int)O, (int)T,
                              (int)N_img, 1, true, filter_img,
                              (cudaStream_t)stream, 0, 1);
}

extern "C" int b200d2_diff2_coarse_cc(const b200d2_view* view, const float* d_trans_x,
                                      const float* d_trans_y, const float* d_corr,
                                      const float* d_real, const float* d_imag,
                                      const float* d_eulers, float* d_diff2s, size_t O,
                                      size_t T, size_t N_img, void* stream, int precision) {
  int st = b200d2::check_common(view, d_trans_x, d_trans_y, d_corr, d_real,
                                d_imag, d_eulers, d_diff2s, O, T, N_img);
  if (st != B200D2_OK) return st;
  if (precision != B200D2_PREC_FP32) return B200D2_ERR_UNSUPPORTED;
  return b200d2::direct_batch(*view, d_eulers, d_trans_x, d_trans_y, d_real,
                              d_imag, d_corr, 0, d_diff2s, 0, (int)O, (int)T,
                              (int)N_img, 1, false, 0, (cudaStream_t)stream, 1, 0);
}

extern "C" int b200d2_diff2_coarse_cc_f64(const b200d2_view* view, const float* d_trans_x,
                                          const float* d_trans_y, const float* d_corr,
                                          const float* d_real, const float* d_imag,
                                          const float* d_eulers, double* d_diff2s, size_t O,
                                          size_t T, size_t N_img, void* stream) {
  int st = b200d2::check_common(view, d_trans_x, d_trans_y, d_corr, d_real,
                                d_imag, d_eulers, d_diff2s, O, T, N_img);
  if (st != B200D2_OK) return st;
  return b200d2::direct_batch(*view, d_eulers, d_trans_x, d_trans_y, d_real,
                              d_imag, d_corr, 0, d_diff2s, 0, (int)O, (int)T,
                              (int)N_img, 1, true, 0, (cudaStream_t)stream, 1, 0);
}
