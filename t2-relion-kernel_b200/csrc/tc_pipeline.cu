// tc_pipeline.cu -- tensor-core coarse pass for a batch of particles.
//
// diff2[p][o][t] = sum_px w|X|^2 + sum_px w|A_o|^2 - 2 Re sum_px (w S_t X_p) conj(A_o)
//                =      normX[p] +       normA[p][o] - 2 cross[(p,t)][o]
// with w = corr/2.  The cross term is a dense complex-as-real contraction:
//   C[m = p*T + t][o] = sum_kk Aop[m][kk] * Bop[o][kk],   kk = 2*pixel + {re, im}
// run on tcgen05 tensor cores with FP32 accumulation in TMEM.  Operands are
// split into hi + lo parts (BF16, FP16 or TF32) and three products are
// accumulated (hi*hi + hi*lo + lo*hi) to recover near-FP32 accuracy, or taken
// once (TF32, FP16); the norms are accumulated in FP64 and the final
// combination is FP64.  The FP16 forms scale each particle's rows and each
// orientation's row by a power of two (largest component in [2^13, 2^14)) and
// divide the scales out exactly in the combine.
//
// Stages (one kernel each):
//   0 pixel_list : in-radius pixel list (FilterCoarseParamImage, src/main.cu:88-151)
//   1 phase      : per-translation separable phase tables e^{i x tx}, e^{i y ty}
//   2 project    : B = projections of every orientation at every listed pixel
//                  (project3Dmodel, src/acc_projectorkernel_impl.h:178-252), split
//                  into hi/lo planes, plus |B|^2
//   3 normx      : sum over all pixels of w|X|^2 per particle (FP64)
//   4 norma      : normX[p] + sum_k w_p(k)|B_o(k)|^2 (FP64)
//   5 gen_a      : A = w * X_p * e^{i(x tx + y ty)} for every (particle, translation)
//                  row (translatePixel, src/cuda_device_utils.cuh:110-129), split
//   6 gemm       : persistent tcgen05 contraction, TMA-fed, double-buffered TMEM
//                  accumulators, fused FP64 combine + store + per-particle argmin
//   7 finalize   : per-particle min / argmin from the packed keys
//
// Score CC (cuda_kernel_diff2_CC_coarse, src/diff2.cuh:691-809): the same
// contraction c = sum (corr/2) Re(S_t conj(A_o)); the norm stage stores
// k[p][o] = -sqrt(2 / sum (corr/2)|A_o|^2) (FP64, and rounded to FP32) in
// place of nA, and the combine writes k c = -sum corr Re(conj(A) S) /
// sqrt(sum corr |A|^2).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "tc_sm100.cuh"

namespace b200d2 {

// ------------------------------------------------------------------ geometry
constexpr int kMaxSplit = 8;  // largest k-split of the single-CTA contraction

struct TcGeom {
  int P, O, T, N_img, K_c, Kpad, Mrows, Mpad, Opad, maxR, exw, eyw;
  int elem, BK, terms;
  int Kq;  // row stride (doubles) of |B|^2 and of the compacted weights: Kpad / 2, zero padded
  // 1: the contraction generates the A operand in shared memory (no A planes
  // in the workspace, no operand-generation stage); 0: A is written to the
  // workspace by tc_gen_a_kernel and read by TMA
  int gen;
  size_t off_status, off_xy, off_idx, off_ex, off_ey, off_ph, off_bhi, off_blo, off_q, off_w, off_normx, off_na, off_nahl,
      off_ahi, off_alo, off_keys, off_sa, off_sb, off_part, off_cnt, off_wx, off_cxy, off_thdr, off_exc, off_eyc, total;
  // device flags read by the projection stage (kEulCheckBlocks words): all
  // 0 = the workspace already holds this call's projections (skip the
  // stage), else project and copy the Euler matrices to d_eul_cache; null =
  // always project (both set by the single-particle entry point's projection
  // cache)
  const int* d_proj_need;
  float* d_eul_cache;
  int split_max;  // largest k-split the workspace holds partial sums for
  int n_cnt;      // split arrival counters
};

static int num_sms();

// Operand mode of the contraction (b200d2_set_operand_gen): 0 (default) = A
// materialised in the workspace by tc_gen_a_kernel and read by TMA, 1 = A
// generated inside the contraction.  At C2 (BF16x3, CTA pairs) the
// generating contraction takes 2.19 ms against 1.67 ms plus 0.09 ms for the
// materialising kernel: its generator warps' shared-memory loads and stores
// add to the tensor cores' operand reads, and shared-memory bandwidth bounds
// it, where TMA writes A without loads.
static std::atomic<int> g_operand_gen{0};

static inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Largest |x| or |y| accepted for caller-listed pixel coordinates.
constexpr int kListedExtent = 512;

// Number of listed pixels and the largest |x| or |y| among them (the extent
// of the phase tables).
static int count_inside(const b200d2_view& v, int N_img, int* extent) {
  int n = 0, r = 0;
  for (int i = 0; i < N_img; ++i) {
    int x = i % v.imgX, y = i / v.imgX;
    if (y > v.maxR) y -= v.imgY;
    if (pixel_maybe_inside(x, y, v.padding_factor, v.maxR2_padded)) {
      ++n;
      r = std::max(r, std::max(x < 0 ? -x : x, y < 0 ? -y : y));
    }
  }
  if (extent) *extent = r;
  return n;
}

// mrows >= 0 overrides the row count (uneven batches: the sum of every
// particle's translations; b.T is then the number of phase tables).
static TcGeom make_geom(const b200d2_view& v, const b200d2_batch& b, int prec, int mrows = -1,
                        bool allow_split = true) {
  TcGeom g;
  memset(&g, 0, sizeof(g));
  g.P = b.P;
  g.O = b.O;
  g.T = b.T;
  g.N_img = b.N_img;
  int extent = 0;
  if (b.d_coor_xy) {
    g.K_c = b.n_listed;  // caller-listed pixels (coordinates are device data)
    extent = kListedExtent;
  } else {
    g.K_c = count_inside(v, b.N_img, &extent);
  }
  g.elem = (prec == B200D2_PREC_TF32 || prec == B200D2_PREC_TF32X3) ? 4 : 2;
  g.BK = 128 / g.elem;
  g.terms = (prec == B200D2_PREC_TF32 || prec == B200D2_PREC_FP16) ? 1 : 3;
  g.Kpad = (int)align_up((size_t)std::max(2 * g.K_c, 1), (size_t)g.BK);
  g.Mrows = mrows >= 0 ? mrows : b.P * b.T;
  g.Mpad = (int)align_up((size_t)g.Mrows, 128);
  g.Opad = (int)align_up((size_t)b.O, 256);
  g.maxR = extent;  // phase tables cover x in [0, extent], y in [-extent, extent]
  g.exw = extent + 1;
  g.eyw = 2 * extent + 1;
  const int planes = g.terms == 3 ? 2 : 1;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes, 1024);
    return at;
  };
  g.off_status = take(256);
  g.off_xy = take(sizeof(int2) * (size_t)std::max(g.K_c, 1));
  g.off_idx = take(sizeof(int) * (size_t)std::max(g.K_c, 1));
  g.off_ex = take(sizeof(float2) * (size_t)g.T * g.exw);
  g.off_ey = take(sizeof(float2) * (size_t)g.T * g.eyw);
  g.off_ph = take(sizeof(float2) * (size_t)g.T * (g.Kpad / 2));  // phase of every (table, listed pixel)
  g.off_bhi = take((size_t)g.Opad * g.Kpad * g.elem);
  g.off_blo = planes == 2 ? take((size_t)g.Opad * g.Kpad * g.elem) : g.off_bhi;
  g.Kq = g.Kpad / 2;  // a multiple of 16
  g.off_q = take(sizeof(double) * (size_t)g.O * g.Kq);
  g.off_w = take(sizeof(double) * (size_t)g.P * g.Kq);
  g.off_normx = take(sizeof(double) * (size_t)g.P);
  g.off_na = take(sizeof(double) * (size_t)g.P * g.O);
  g.off_nahl = take(sizeof(float2) * (size_t)g.P * g.O);  // nA as an unevaluated sum hi + lo of two floats
  g.gen = g_operand_gen.load();
  if (g.gen) {  // no A planes: the contraction writes A into shared memory
    g.off_ahi = g.off_alo = 0;
  } else {
    g.off_ahi = take((size_t)g.Mpad * g.Kpad * g.elem);
    g.off_alo = planes == 2 ? take((size_t)g.Mpad * g.Kpad * g.elem) : g.off_ahi;
  }
  // weighted images w X of the listed pixels [P][Kpad / 2] (FP16 forms: times
  // the particle scale), read by the contraction's operand generation
  g.off_wx = take(sizeof(float2) * (size_t)(g.P + 1) * (g.Kpad / 2));  // + an all-zero row (rows past the batch)
  // phase tables deduplicated by translation value: table -> (x row, y row),
  // a header {rows x, rows y, extent, fits}, and the compact rows
  g.off_cxy = take(sizeof(int2) * (size_t)std::max(g.T, 1));
  g.off_thdr = take(4 * sizeof(int));
  g.off_exc = take(sizeof(float2) * (size_t)g.T * g.exw);
  g.off_eyc = take(sizeof(float2) * (size_t)g.T * g.eyw);
  g.off_keys = take(sizeof(unsigned long long) * (size_t)g.P);
  g.off_sa = take(sizeof(float) * (size_t)g.P);     // FP16 forms: 1 / particle scale
  g.off_sb = take(sizeof(float) * (size_t)g.Opad);  // FP16 forms: 1 / orientation scale
  // split-K: partial sums when the 256-wide tiles do not fill the GPU (the
  // 128-wide tiling needs the same bytes: twice the tiles, half the width)
  {
    const int mt = g.Mpad / 128, tiles256 = mt * (g.Opad / 256);
    const int kb = g.Kpad / g.BK;  // k-blocks of the 128-byte rows (fewest)
    g.split_max = 1;
    const int sms = num_sms();
    if (allow_split && tiles256 < sms)
      while (g.split_max * 2 <= kMaxSplit && (long long)tiles256 * g.split_max * 2 <= 2LL * sms && kb / (g.split_max * 2) >= 2)
        g.split_max *= 2;
    g.off_part = take(g.split_max > 1 ? (size_t)g.split_max * tiles256 * 256 * 128 * sizeof(float) : 0);
    g.n_cnt = 8 * mt * (g.Opad / 128);  // per (tile, column half, lane quadrant) of 128-wide tiles
    g.off_cnt = take(sizeof(unsigned) * (size_t)g.n_cnt);
  }
  g.total = o;
  return g;
}

// Per-particle description for uneven batches (device resident, built by a
// plan).  Uniform batches pass no table and use base pointer + p * stride.
struct PartDev {
  const float* re;
  const float* im;
  const float* corr;
  float* out;      // [O][T] of this particle
  const int* inv;  // [O_all] -> index in this particle's orientation list, or -1
  int T, O, row0, pad;
};

// Device tables of an uneven batch, owned by a plan.
struct UnevenTabs {
  const PartDev* parts;   // [P]
  const int4* rows;       // [Mrows]
  const int2* tiles[3];   // work lists: 128 x 256, 128 x 128 and (CTA pairs) 256 x 256 tiles
  int ntiles[3];
  const float2* tab_txy;  // [ntab] translation of each phase table
  int ntab;
  int Mrows;
  // the norm kernel's work lists (64-, 32- and 16-particle tiles by 64
  // orientations) over the particle order nperm (null: 0 .. P-1), and the
  // list in use (-1: the first whose tiles give every SM a CTA)
  const int2* ntile[3];
  int nntile[3];
  const int* nperm;
  int nsel;
};

// Optional tables of an uneven batch; all null for a uniform batch.
struct Layout {
  const PartDev* parts;  // [P]
  const int4* rows;      // [Mrows]: (particle, translation, phase table, 0)
  const int2* tiles;     // [ntiles]: (m tile, n tile) that some particle needs
  int ntiles;
};

template <typename T>
static inline T* ws_at(void* ws, size_t off) {
  return reinterpret_cast<T*>(reinterpret_cast<uint8_t*>(ws) + off);
}

// ------------------------------------------------------------------ stage 0
__global__ void __launch_bounds__(1024) tc_pixel_list_kernel(b200d2_view v, int N_img, int2* xy,
                                                             int* idx, uint32_t* status,
                                                             unsigned long long* keys, int P,
                                                             const float* __restrict__ coor_xy,
                                                             int n_listed, int ext, unsigned* cnt, int n_cnt) {
  __shared__ int s_cnt[32];
  __shared__ int s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    *status = 0;
    s_base = 0;
  }
  for (int p = tid; p < P; p += blockDim.x) keys[p] = ~0ull;
  for (int i = tid; i < n_cnt; i += blockDim.x) cnt[i] = 0u;  // split-K arrival counters
  __syncthreads();  // the status reset above precedes any report below
  if (coor_xy) {  // caller-listed pixels, in the caller's order
    bool bad = false;
    for (int k = tid; k < n_listed; k += blockDim.x) {
      const float fx = coor_xy[2 * k], fy = coor_xy[2 * k + 1];
      const int x = clampi(__float2int_rn(fx), 0, ext);
      const int y = clampi(__float2int_rn(fy), -ext, ext);
      // outside the documented range, or not integer-valued: report it (the
      // scores of this call are then not those of the listed pixels)
      bad |= (float)x != fx || (float)y != fy;
      xy[k] = make_int2(x, y);
      idx[k] = k;
    }
    if (__syncthreads_or(bad) && tid == 0) atomicCAS(status, 0u, (uint32_t)B200D2_ERR_INVALID);
    return;
  }
  for (int base = 0; base < N_img; base += 1024) {
    const int i = base + tid;
    int x = 0, y = 0;
    bool in = false;
    if (i < N_img) {
      pixel_coor(i, v.imgX, v.imgY, v.maxR, x, y);
      in = pixel_maybe_inside(x, y, v.padding_factor, v.maxR2_padded);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    if (lane == 0) s_cnt[warp] = __popc(bal);
    __syncthreads();
    int off = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
      const int c = s_cnt[w];
      off += (w < warp) ? c : 0;
      total += c;
    }
    if (in) {
      const int slot = s_base + off + __popc(bal & ((1u << lane) - 1u));
      xy[slot] = make_int2(x, y);
      idx[slot] = i;
    }
    __syncthreads();
    if (tid == 0) s_base += total;
    __syncthreads();
  }
}

// ------------------------------------------------------------------ stage 1
// T phase tables (one per translation).  With `txy` given, ntab tables whose
// translation is txy[tab] (uneven batches: one table per distinct
// translation of every particle); otherwise table t uses (tx[t], ty[t]).
__global__ void tc_phase_kernel(const float* __restrict__ tx, const float* __restrict__ ty, int T,
                                int maxR, float2* ex, float2* ey, const float2* __restrict__ txy) {
  const int exw = maxR + 1, eyw = 2 * maxR + 1;
  const int n1 = T * exw, n2 = T * eyw;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2; i += gridDim.x * blockDim.x) {
    double s, c;
    if (i < n1) {
      const int t = i / exw, x = i % exw;
      const float sx = txy ? txy[t].x : tx[t];
      sincos((double)x * (double)sx, &s, &c);
      ex[i] = make_float2((float)c, (float)s);
    } else {
      const int j = i - n1, t = j / eyw, y = j % eyw - maxR;
      const float sy = txy ? txy[t].y : ty[t];
      sincos((double)y * (double)sy, &s, &c);
      ey[j] = make_float2((float)c, (float)s);
    }
  }
}

// Phase of every (table, listed pixel) as the product of the separable
// tables, ph[t][kp] = e^{i x tx} e^{i y ty} (zero past K_c), so that stage 5
// reads one coalesced 8-byte value per element of A.
__global__ void tc_phase2d_kernel(const float2* __restrict__ ex, const float2* __restrict__ ey,
                                  const int2* __restrict__ xy, int K_c, int Kh, int T, int maxR, float2* ph) {
  const int kp = blockIdx.x * blockDim.x + threadIdx.x;
  if (kp >= Kh) return;
  const int exw = maxR + 1, eyw = 2 * maxR + 1;
  int2 c = make_int2(0, 0);
  if (kp < K_c) c = xy[kp];
  for (int t = blockIdx.y; t < T; t += gridDim.y) {
    float2 v = make_float2(0.f, 0.f);
    if (kp < K_c) {
      const float2 fx = ex[t * exw + c.x];
      const float2 fy = ey[t * eyw + c.y + maxR];
      v = make_float2(__fmaf_rn(fx.x, fy.x, -__fmul_rn(fx.y, fy.y)), __fmaf_rn(fx.x, fy.y, __fmul_rn(fx.y, fy.x)));
    }
    ph[(size_t)t * Kh + kp] = v;
  }
}

// Phase tables deduplicated by translation value, for the contraction's
// operand generation.  e^{i x tx} depends only on tx and e^{i y ty} only on
// ty, and translation grids repeat few values (a disc of radius 6 px has 113
// translations but 13 distinct tx and 13 distinct ty), so the rows of the
// per-table tables ex / ey that belong to equal values (bit for bit) are kept
// once: cxy[t] = (x row, y row) of table t, exc [rows x][ext + 1] and
// eyc [rows y][2 ext + 1], with ext the largest |x| or |y| of the listed
// pixels.  hdr = {rows x, rows y, ext, fits}: fits = 1 when the compact rows
// take at most `cap` entries (they then fit the contraction's shared-memory
// table; otherwise it reads the (table, pixel) products ph from global
// memory).  The values are copies of ex / ey, so both give bit-identical
// operands.  One CTA of kCompactThreads threads; up to kCompactMaxT tables.
constexpr int kCompactThreads = 1024, kCompactMaxT = 4096;
__global__ void __launch_bounds__(kCompactThreads) tc_phase_compact_kernel(
    const float* __restrict__ tx, const float* __restrict__ ty, const float2* __restrict__ txy, int T,
    const int2* __restrict__ xy, int K_c, const float2* __restrict__ ex, const float2* __restrict__ ey, int maxR,
    int2* __restrict__ cxy, int* __restrict__ hdr, float2* __restrict__ exc, float2* __restrict__ eyc, int cap) {
  __shared__ int s_fx[kCompactMaxT], s_fy[kCompactMaxT];  // first table with the same value; then its row
  __shared__ int s_part[2][kCompactThreads / 32];
  __shared__ int s_ext, s_n[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_ext = 0;
  __syncthreads();
  int e = 0;
  for (int k = tid; k < K_c; k += kCompactThreads) {
    const int2 c = xy[k];
    e = max(e, max(abs(c.x), abs(c.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (lane == 0) atomicMax(&s_ext, e);
  __syncthreads();
  const int ext = min(s_ext, maxR);
  if (T > kCompactMaxT) {  // too many tables to deduplicate here: global products
    if (tid == 0) {
      hdr[0] = hdr[1] = 0;
      hdr[2] = ext;
      hdr[3] = 0;
    }
    return;
  }
  auto val = [&](int t, int axis) -> uint32_t {
    const float v = txy ? (axis ? txy[t].y : txy[t].x) : (axis ? ty[t] : tx[t]);
    return __float_as_uint(v);
  };
  for (int t = tid; t < T; t += kCompactThreads) {
    const uint32_t vx = val(t, 0), vy = val(t, 1);
    int fx = t, fy = t;
    for (int u = 0; u < t && (fx == t || fy == t); ++u) {
      if (fx == t && val(u, 0) == vx) fx = u;
      if (fy == t && val(u, 1) == vy) fy = u;
    }
    s_fx[t] = fx;
    s_fy[t] = fy;
  }
  __syncthreads();
  // rank of every first occurrence among the first occurrences: each thread
  // counts a contiguous chunk of tables, then an exclusive scan over threads
  const int chunk = (T + kCompactThreads - 1) / kCompactThreads;
  const int t0 = min(T, tid * chunk), t1 = min(T, t0 + chunk);
  int nx = 0, ny = 0;
  for (int t = t0; t < t1; ++t) {
    nx += s_fx[t] == t;
    ny += s_fy[t] == t;
  }
  int ix = nx, iy = ny;  // inclusive scan within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ax = __shfl_up_sync(0xffffffffu, ix, o), ay = __shfl_up_sync(0xffffffffu, iy, o);
    if (lane >= o) {
      ix += ax;
      iy += ay;
    }
  }
  if (lane == 31) {
    s_part[0][warp] = ix;
    s_part[1][warp] = iy;
  }
  __syncthreads();
  if (tid == 0) {
    int ax = 0, ay = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) {
      const int bx = s_part[0][w], by = s_part[1][w];
      s_part[0][w] = ax;
      s_part[1][w] = ay;
      ax += bx;
      ay += by;
    }
    s_n[0] = ax;
    s_n[1] = ay;
  }
  __syncthreads();
  int rx = s_part[0][warp] + ix - nx, ry = s_part[1][warp] + iy - ny;  // exclusive
  // turn first occurrences into their row numbers (other entries keep the
  // index of their first occurrence, which is below them)
  for (int t = t0; t < t1; ++t) {
    if (s_fx[t] == t) s_fx[t] = -1 - rx++;
    if (s_fy[t] == t) s_fy[t] = -1 - ry++;
  }
  __syncthreads();
  const int nrx = s_n[0], nry = s_n[1];
  const int ew = ext + 1, yw = 2 * ext + 1;
  const bool fits = (long long)nrx * ew + (long long)nry * yw <= cap;
  const int exw = maxR + 1, eyw = 2 * maxR + 1;
  for (int t = tid; t < T; t += kCompactThreads) {
    const int fx = s_fx[t], fy = s_fy[t];
    const int rxt = fx < 0 ? -1 - fx : -1 - s_fx[fx];
    const int ryt = fy < 0 ? -1 - fy : -1 - s_fy[fy];
    cxy[t] = make_int2(rxt, ryt);
    if (fits) {
      if (fx < 0)
        for (int x = 0; x <= ext; ++x) exc[rxt * ew + x] = ex[(size_t)t * exw + x];
      if (fy < 0)
        for (int y = -ext; y <= ext; ++y) eyc[ryt * yw + y + ext] = ey[(size_t)t * eyw + y + maxR];
    }
  }
  if (tid == 0) {
    hdr[0] = nrx;
    hdr[1] = nry;
    hdr[2] = ext;
    hdr[3] = fits ? 1 : 0;
  }
}

// ------------------------------------------------------------------ splits
__device__ __forceinline__ float tf32_round(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

template <int PREC>
__device__ __forceinline__ void store_split(void* hi, void* lo, size_t at, float re, float im) {
  if constexpr (PREC == B200D2_PREC_BF16X3) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
    reinterpret_cast<__nv_bfloat162*>(hi)[at] = h;
    reinterpret_cast<__nv_bfloat162*>(lo)[at] = l;
  } else if constexpr (PREC == B200D2_PREC_FP16X3) {
    const __half2 h = __floats2half2_rn(re, im);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(re - hf.x, im - hf.y);
    reinterpret_cast<__half2*>(hi)[at] = h;
    reinterpret_cast<__half2*>(lo)[at] = l;
  } else if constexpr (PREC == B200D2_PREC_FP16) {
    reinterpret_cast<__half2*>(hi)[at] = __floats2half2_rn(re, im);
  } else if constexpr (PREC == B200D2_PREC_TF32X3) {
    const float hr = tf32_round(re), hm = tf32_round(im);
    reinterpret_cast<float2*>(hi)[at] = make_float2(hr, hm);
    reinterpret_cast<float2*>(lo)[at] = make_float2(tf32_round(re - hr), tf32_round(im - hm));
  } else {
    reinterpret_cast<float2*>(hi)[at] = make_float2(tf32_round(re), tf32_round(im));
  }
}

// Four consecutive complex values at element `at` (a multiple of 4): the
// same values as four store_split calls, written as 16-byte stores.
template <int PREC>
__device__ __forceinline__ void store_split4(void* hi, void* lo, size_t at, const float (&re)[4],
                                             const float (&im)[4]) {
  if constexpr (PREC == B200D2_PREC_BF16X3 || PREC == B200D2_PREC_FP16X3 || PREC == B200D2_PREC_FP16) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if constexpr (PREC == B200D2_PREC_BF16X3) {
        const __nv_bfloat162 hv = __floats2bfloat162_rn(re[j], im[j]);
        const float2 hf = __bfloat1622float2(hv);
        const __nv_bfloat162 lv = __floats2bfloat162_rn(re[j] - hf.x, im[j] - hf.y);
        h[j] = *reinterpret_cast<const uint32_t*>(&hv);
        l[j] = *reinterpret_cast<const uint32_t*>(&lv);
      } else {
        const __half2 hv = __floats2half2_rn(re[j], im[j]);
        const float2 hf = __half22float2(hv);
        const __half2 lv = __floats2half2_rn(re[j] - hf.x, im[j] - hf.y);
        h[j] = *reinterpret_cast<const uint32_t*>(&hv);
        l[j] = *reinterpret_cast<const uint32_t*>(&lv);
      }
    }
    reinterpret_cast<uint4*>(reinterpret_cast<uint32_t*>(hi) + at)[0] = make_uint4(h[0], h[1], h[2], h[3]);
    if constexpr (PREC != B200D2_PREC_FP16)
      reinterpret_cast<uint4*>(reinterpret_cast<uint32_t*>(lo) + at)[0] = make_uint4(l[0], l[1], l[2], l[3]);
  } else {
    float hr[4], hm[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      hr[j] = tf32_round(re[j]);
      hm[j] = tf32_round(im[j]);
    }
    float4* ph = reinterpret_cast<float4*>(reinterpret_cast<float2*>(hi) + at);
    ph[0] = make_float4(hr[0], hm[0], hr[1], hm[1]);
    ph[1] = make_float4(hr[2], hm[2], hr[3], hm[3]);
    if constexpr (PREC == B200D2_PREC_TF32X3) {
      float4* pl = reinterpret_cast<float4*>(reinterpret_cast<float2*>(lo) + at);
      pl[0] = make_float4(tf32_round(re[0] - hr[0]), tf32_round(im[0] - hm[0]), tf32_round(re[1] - hr[1]),
                          tf32_round(im[1] - hm[1]));
      pl[1] = make_float4(tf32_round(re[2] - hr[2]), tf32_round(im[2] - hm[2]), tf32_round(re[3] - hr[3]),
                          tf32_round(im[3] - hm[3]));
    }
  }
}

// ------------------------------------------------------------------ stage 2
// A CTA takes kProjOrients consecutive orientations of one block of pixels,
// one orientation after the other: consecutive orientations are usually
// in-plane rotations of one viewing direction, which sample the same slice of
// the volume, so the block's texels are reused from L1.
constexpr int kProjOrients = 8;  // divides Opad (a multiple of 256)
template <int PREC>
__global__ void __launch_bounds__(128) tc_project_kernel(b200d2_view v, const float* __restrict__ eulers,
                                                         int O, const int2* __restrict__ xy, int K_c,
                                                         int Kpad, void* bhi, void* blo, double* q,
                                                         const int* __restrict__ need, float* eul_cache) {
  if (need) {  // kEulCheckBlocks verdict words of the cache check
    const int any = __syncthreads_or(threadIdx.x < kEulCheckBlocks ? need[threadIdx.x] : 0);
    if (!any) return;     // the workspace holds these projections already
    if (blockIdx.x == 0)  // keep the Euler matrices projected here for the next call's check
      for (int i = threadIdx.x; i < kProjOrients * 9; i += blockDim.x) {
        const int o = blockIdx.y * kProjOrients + i / 9;
        if (o < O) eul_cache[(size_t)o * 9 + i % 9] = eulers[(size_t)o * 9 + i % 9];
      }
  }
  const int kp = blockIdx.x * blockDim.x + threadIdx.x;  // complex pixel slot
  if (kp >= Kpad / 2) return;
  const int2 c = kp < K_c ? xy[kp] : make_int2(0, 0);
  for (int j = 0; j < kProjOrients; ++j) {
    const int o = blockIdx.y * kProjOrients + j;
    float2 b = make_float2(0.f, 0.f);
    if (o < O && kp >= K_c) q[(size_t)o * (Kpad / 2) + kp] = 0.0;  // zero padding of the |B|^2 row
    if (o < O && kp < K_c) {
      float e[6];
      const float* eo = eulers + (size_t)o * 9;
      e[0] = eo[0];
      e[1] = eo[1];
      e[2] = eo[3];
      e[3] = eo[4];
      e[4] = eo[6];
      e[5] = eo[7];
      b = project_pixel(v, (float)c.x, (float)c.y, e);
      q[(size_t)o * (Kpad / 2) + kp] = (double)b.x * (double)b.x + (double)b.y * (double)b.y;
    }
    store_split<PREC>(bhi, blo, (size_t)o * (Kpad / 2) + kp, b.x, b.y);
  }
}

// ------------------------------------------------------------------ FP16 scales
// Exponent e with max_abs * 2^e in [2^13, 2^14) (0 for a zero or non-finite
// maximum), clamped so that 2^e and 2^-e are normal FP32 numbers.
__device__ __forceinline__ int pow2_scale_exp(float max_abs) {
  if (!(max_abs > 0.f) || !isfinite(max_abs)) return 0;
  int e;
  frexpf(max_abs, &e);  // max_abs = f * 2^e, f in [0.5, 1)
  return max(-100, min(100, 14 - e));
}

// Maximum over a CTA of blockDim.x <= 1024 threads; every thread gets it.
__device__ __forceinline__ float block_max(float v) {
  __shared__ float s_part[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_part[warp] = v;
  __syncthreads();
  float m = 0.f;
  for (int w = 0; w < nw; ++w) m = fmaxf(m, s_part[w]);
  return m;
}

// FP16 forms, stage 2: one CTA per orientation.  Pass 1 projects every listed
// pixel, writes |B|^2 and takes the largest component; pass 2 projects again
// (same inputs, same bits) and stores the split of the scaled projection.
// inv_sb[o] = 2^-e is divided out in the combine.
template <int PREC>
__global__ void __launch_bounds__(256) tc_project_scaled_kernel(b200d2_view v, const float* __restrict__ eulers,
                                                                int O, const int2* __restrict__ xy, int K_c,
                                                                int Kpad, void* bhi, void* blo, double* q,
                                                                float* inv_sb) {
  const int o = blockIdx.x, half = Kpad / 2;
  float e[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (o < O) {
    const float* eo = eulers + (size_t)o * 9;
    e[0] = eo[0];
    e[1] = eo[1];
    e[2] = eo[3];
    e[3] = eo[4];
    e[4] = eo[6];
    e[5] = eo[7];
  }
  float mx = 0.f;
  if (o < O)
    for (int kp = threadIdx.x; kp < K_c; kp += blockDim.x) {
      const int2 c = xy[kp];
      const float2 b = project_pixel(v, (float)c.x, (float)c.y, e);
      q[(size_t)o * half + kp] = (double)b.x * (double)b.x + (double)b.y * (double)b.y;
      mx = fmaxf(mx, fmaxf(fabsf(b.x), fabsf(b.y)));
    }
  if (o < O)
    for (int kp = K_c + threadIdx.x; kp < half; kp += blockDim.x) q[(size_t)o * half + kp] = 0.0;
  const int ex = pow2_scale_exp(block_max(mx));
  const float sc = ldexpf(1.f, ex);
  if (threadIdx.x == 0) inv_sb[o] = ldexpf(1.f, -ex);
  for (int kp = threadIdx.x; kp < half; kp += blockDim.x) {
    float2 b = make_float2(0.f, 0.f);
    if (o < O && kp < K_c) {
      const int2 c = xy[kp];
      b = project_pixel(v, (float)c.x, (float)c.y, e);
    }
    store_split<PREC>(bhi, blo, (size_t)o * half + kp, b.x * sc, b.y * sc);
  }
}

// FP16 forms, stage 1: per-particle scale of the A rows.  A component of a
// row is fma(w re, c, -(w im) s) or fma(w re, s, (w im) c) with |c|, |s| <= 1,
// so |w re| + |w im| bounds it; inv_sa[p] = 2^-e of that bound's maximum.
__global__ void __launch_bounds__(256) tc_scale_a_kernel(const float* __restrict__ re,
                                                         const float* __restrict__ im,
                                                         const float* __restrict__ corr, long long stride,
                                                         const PartDev* __restrict__ parts,
                                                         const int* __restrict__ idx, int K_c, float* inv_sa) {
  const long long p = blockIdx.x;
  const float* pre = parts ? parts[p].re : re + p * stride;
  const float* pim = parts ? parts[p].im : im + p * stride;
  const float* pco = parts ? parts[p].corr : corr + p * stride;
  float mx = 0.f;
  for (int k = threadIdx.x; k < K_c; k += blockDim.x) {
    const int pix = idx[k];
    const float w = pco[pix] / 2;
    mx = fmaxf(mx, fabsf(w * pre[pix]) + fabsf(w * pim[pix]));
  }
  // 2^-20 of headroom for the rounding of the phase factors
  const int ex = pow2_scale_exp(block_max(mx) * (1.f + 0x1p-20f));
  if (threadIdx.x == 0) inv_sa[p] = ldexpf(1.f, -ex);
}

// ------------------------------------------------------------------ stage 3
__global__ void __launch_bounds__(256) tc_normx_kernel(const float* __restrict__ re,
                                                       const float* __restrict__ im,
                                                       const float* __restrict__ corr,
                                                       long long stride, int N_img, double* normx,
                                                       const PartDev* __restrict__ parts,
                                                       const int* __restrict__ idx, int K_c, int Kq,
                                                       double* wcomp, float2* wx, const float* __restrict__ inv_sa) {
  const long long p = blockIdx.x;
  const float* pre = parts ? parts[p].re : re + p * stride;
  const float* pim = parts ? parts[p].im : im + p * stride;
  const float* pco = parts ? parts[p].corr : corr + p * stride;
  // the weights of the listed pixels, compacted for the normA contraction
  // (Kq = Kpad / 2 entries per particle), and the weighted image w X of the
  // listed pixels for the contraction's operand generation: w = corr / 2,
  // (w re, w im), then times the FP16 forms' particle scale, rounded as the
  // materialised operand's generation rounds them
  const float sc = inv_sa ? __frcp_rn(inv_sa[p]) : 1.f;
  for (int k = threadIdx.x; k < Kq; k += blockDim.x) {
    double wd = 0.0;
    float2 v = make_float2(0.f, 0.f);
    if (k < K_c) {
      const int pix = idx[k];
      const float w = pco[pix] / 2;
      wd = (double)pco[pix] / 2.0;
      v = make_float2(w * pre[pix], w * pim[pix]);
      if (inv_sa) {
        v.x *= sc;
        v.y *= sc;
      }
    }
    wcomp[p * Kq + k] = wd;
    wx[p * Kq + k] = v;
    if (p == 0) wx[(long long)gridDim.x * Kq + k] = make_float2(0.f, 0.f);  // the zero row after the last particle
  }
  double acc = 0.0;
  for (int i = threadIdx.x; i < N_img; i += blockDim.x) {
    const double r = pre[i], m = pim[i];
    acc += (r * r + m * m) * ((double)pco[i] / 2.0);
  }
  __shared__ double s[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += s[w];
    normx[p] = t;
  }
}

// ------------------------------------------------------------------ stage 4
// na[p][o] = normX[p] + sum_k w_p(k) |B_o(k)|^2, FP64 products and sums.
// The weights w[p][k] and |B|^2 q[o][k] arrive as FP64 rows (written by the
// normX and projector stages).  The product runs on the FP64 tensor-core
// MMA (mma.sync m8n8k4 f64: FP64 operands, products and sums); the k dimension
// is walked in 16-pixel slabs copied into shared memory with cp.async,
// double-buffered so the next slab's loads overlap this slab's MMAs.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sm100::smem_u32(smem)), "l"(gmem),
               "r"(pred ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sm100::smem_u32(smem)), "l"(gmem),
               "r"(pred ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// FP64 tensor-core MMA (DMMA): D[8x8] += A[8x4] * B[4x8], all FP64.  Lane l
// holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// CTA tile: (2*8*WM) particles x (2*8*WN) orientations, 4 warps in a 2 x 2
// grid, each warp WM x WN DMMA tiles of 8 x 8 (WN = 4 unless the batch is too
// small to give every SM a CTA); 32-pixel slabs in a three-stage
// cp.async ring (one barrier per slab, two slabs in flight).  (Splitting each
// slab's pixels over two groups of 4 warps, with the two sums added at the
// end, measured slower: 94.9 against 86.3 us at 128 particles.)
// cc: store k = -sqrt(2 / sum w|B|^2) (the CC score's factor) instead of nA.
constexpr int kNormaKC = 32, kNormaLD = kNormaKC + 4, kNormaStages = 3;
template <int WM, int WN>
constexpr size_t norma_smem_bytes() {
  return sizeof(double) * kNormaStages * (16 * WM + 16 * WN) * kNormaLD;
}

constexpr int kNormaThreads = 128;
template <int WM, int WN, bool LIST>
__global__ void __launch_bounds__(kNormaThreads) tc_norma_kernel(const double* __restrict__ wcomp, int Kq,
                                                       const double* __restrict__ q, int O, int P,
                                                       const double* __restrict__ normx, double* na,
                                                       float2* na_hl, int cc, long long ld,
                                                       const int2* __restrict__ tiles,
                                                       const int* __restrict__ pperm) {
  // Kq: row stride of wcomp and q, a multiple of 16, zero padded; ld: row
  // stride of na and na_hl.  Uneven batches pass a work list `tiles` of
  // (particle tile, orientation tile) pairs that some particle needs, one per
  // CTA, with particle tiles over the order pperm (null: 0 .. P-1); the last
  // slab is zero-filled past Kq.  Shared rows padded to 36 doubles (288 B,
  // 16-byte aligned): the fragment loads of a half-warp (rows g, columns t,
  // g, t < 4) fall on distinct bank pairs 4g + t (mod 16).
  constexpr int KC = kNormaKC, LD = kNormaLD, NST = kNormaStages, CP = 16 * WM, CO = 16 * WN;
  extern __shared__ __align__(16) double norma_smem[];
  double* sw = norma_smem;                   // [NST][CP][LD]
  double* sq = norma_smem + NST * CP * LD;   // [NST][CO][LD]
  constexpr int NT = kNormaThreads;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int wp0 = (warp >> 1) * 8 * WM, wo0 = (warp & 1) * 8 * WN;
  int p0, o0;
  if (LIST) {
    const int2 tl = tiles[blockIdx.x];
    p0 = tl.x * CP;
    o0 = tl.y * CO;
  } else {
    p0 = blockIdx.y * CP;
    o0 = blockIdx.x * CO;
  }
  auto prow = [&](int pl) { return (LIST && pperm) ? pperm[pl] : pl; };  // pl < P
  double acc[WM][WN][2];
#pragma unroll
  for (int i = 0; i < WM; ++i)
#pragma unroll
    for (int j = 0; j < WN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  auto stage = [&](int buf, int k0) {
    // 16-byte pieces (two doubles); rows past P or O and columns past Kq are zero-filled
    double* dw = sw + buf * CP * LD;
    double* dq = sq + buf * CO * LD;
    for (int e = tid; e < CP * (KC / 2); e += NT) {
      const int pp = e / (KC / 2), k = 2 * (e % (KC / 2));
      const bool ok = p0 + pp < P && k0 + k < Kq;
      cp_async16(dw + pp * LD + k, ok ? wcomp + (size_t)prow(p0 + pp) * Kq + k0 + k : wcomp, ok);
    }
    for (int e = tid; e < CO * (KC / 2); e += NT) {
      const int oo = e / (KC / 2), k = 2 * (e % (KC / 2));
      const bool ok = o0 + oo < O && k0 + k < Kq;
      cp_async16(dq + oo * LD + k, ok ? q + (size_t)(o0 + oo) * Kq + k0 + k : q, ok);
    }
  };
  const int nslab = (Kq + KC - 1) / KC;
  // one commit group per slab (empty past the end), so wait<NST-2> leaves
  // exactly the current slab complete
#pragma unroll
  for (int sl = 0; sl < NST - 1; ++sl) {
    if (sl < nslab) stage(sl, sl * KC);
    cp_async_commit();
  }
  for (int sl = 0; sl < nslab; ++sl) {
    cp_async_wait<NST - 2>();
    __syncthreads();  // slab sl visible to all; every warp is done with slab sl - 1
    if (sl + NST - 1 < nslab) stage((sl + NST - 1) % NST, (sl + NST - 1) * KC);
    cp_async_commit();
    const double* cw = sw + (sl % NST) * CP * LD;
    const double* cq = sq + (sl % NST) * CO * LD;
#pragma unroll
    for (int k4 = 0; k4 < KC; k4 += 4) {
      double a[WM], bq[WN];
#pragma unroll
      for (int i = 0; i < WM; ++i) a[i] = cw[(wp0 + 8 * i + gid) * LD + k4 + tig];
#pragma unroll
      for (int j = 0; j < WN; ++j) bq[j] = cq[(wo0 + 8 * j + gid) * LD + k4 + tig];
#pragma unroll
      for (int i = 0; i < WM; ++i)
#pragma unroll
        for (int j = 0; j < WN; ++j) dmma_8x8x4(acc[i][j], a[i], bq[j]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < WM; ++i) {
    const int pl = p0 + wp0 + 8 * i + gid;
    if (pl >= P) continue;
    const int p = prow(pl);
#pragma unroll
    for (int j = 0; j < WN; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int o = o0 + wo0 + 8 * j + 2 * tig + h;
        if (o < O) {
          if (cc) {
            const double k = -sqrt(2.0 / acc[i][j][h]);
            na[(size_t)p * ld + o] = k;
            na_hl[(size_t)p * ld + o] = make_float2((float)k, 0.f);
          } else {
            const double v = normx[p] + acc[i][j][h];
            na[(size_t)p * ld + o] = v;
            const float hi = (float)v;  // v = hi + lo to 48 bits: the combine's double-float operand
            na_hl[(size_t)p * ld + o] = make_float2(hi, (float)(v - (double)hi));
          }
        }
      }
  }
}

template <int WM, int WN>
static cudaError_t launch_norma(cudaStream_t s, const double* wcomp, int Kq, const double* q, int O, int P,
                                const double* normx, double* na, float2* na_hl, int cc, long long ld,
                                const int2* tiles = nullptr, int ntiles = 0, const int* pperm = nullptr) {
  // above 48 KB of dynamic shared memory, per device
  static std::atomic<unsigned long long> opted{0}, opted_list{0};
  if (tiles) {
    const cudaError_t e = smem_opt_in(tc_norma_kernel<WM, WN, true>, (int)norma_smem_bytes<WM, WN>(), opted_list);
    if (e != cudaSuccess) return e;
    if (ntiles == 0) return cudaSuccess;
    tc_norma_kernel<WM, WN, true><<<ntiles, kNormaThreads, norma_smem_bytes<WM, WN>(), s>>>(
        wcomp, Kq, q, O, P, normx, na, na_hl, cc, ld, tiles, pperm);
    return cudaSuccess;
  }
  const cudaError_t e = smem_opt_in(tc_norma_kernel<WM, WN, false>, (int)norma_smem_bytes<WM, WN>(), opted);
  if (e != cudaSuccess) return e;
  const dim3 grid((O + 16 * WN - 1) / (16 * WN), (P + 16 * WM - 1) / (16 * WM));
  tc_norma_kernel<WM, WN, false><<<grid, kNormaThreads, norma_smem_bytes<WM, WN>(), s>>>(
      wcomp, Kq, q, O, P, normx, na, na_hl, cc, ld, nullptr, nullptr);
  return cudaSuccess;
}

// Work lists of the norm kernel for an uneven batch, one per particle-tile
// height (64, 32, 16 particles; 64 orientations wide): the (particle tile,
// orientation tile) pairs in which some particle of the tile needs some
// column of the tile.  need(pl, blk) says whether the pl-th particle of the
// order needs 128-column block blk.
template <class Need>
static void norma_lists(int P, int O, Need need, std::vector<int2> (&lists)[3]) {
  const int nb = (O + 127) / 128, no = (O + 63) / 64;
  for (int li = 0; li < 3; ++li) {
    const int cp = 64 >> li;
    lists[li].clear();
    std::vector<char> un(nb);
    for (int pt = 0; pt < (P + cp - 1) / cp; ++pt) {
      std::fill(un.begin(), un.end(), 0);
      for (int pl = pt * cp; pl < std::min(P, pt * cp + cp); ++pl)
        for (int b = 0; b < nb; ++b) un[b] |= need(pl, b);
      for (int ot = 0; ot < no; ++ot)
        if (un[ot / 2]) lists[li].push_back(make_int2(pt, ot));
    }
  }
}

// ------------------------------------------------------------------ stage 5
// Row m = p*T + t of the translated, weighted image: a = (corr/2) X e^{i(x tx + y ty)},
// the phase read from the (table, pixel) product ph.  A thread writes four
// consecutive complex values of kGenRows consecutive rows with 16-byte
// stores; rows past Mrows are zero.
constexpr int kGenV = 4, kGenRows = 16;
template <int PREC, bool UNEVEN>
__global__ void __launch_bounds__(256) tc_gen_a_kernel(
    const float* __restrict__ re, const float* __restrict__ im, const float* __restrict__ corr,
    long long stride, const int* __restrict__ idx, int K_c, int Kh, const float2* __restrict__ ph, int T,
    int Mrows, void* ahi, void* alo, const PartDev* __restrict__ parts, const int4* __restrict__ rows,
    const float* __restrict__ inv_sa) {
  const int kp0 = (blockIdx.x * blockDim.x + threadIdx.x) * kGenV;
  if (kp0 >= Kh) return;
  int pix[kGenV];
#pragma unroll
  for (int j = 0; j < kGenV; ++j) pix[j] = kp0 + j < K_c ? idx[kp0 + j] : -1;
  const int m0 = blockIdx.y * kGenRows;
  int p = UNEVEN ? 0 : m0 / T;
  int t = UNEVEN ? 0 : m0 - p * T;
  int cur_p = -1;
  float wr[kGenV], wi[kGenV];
#pragma unroll
  for (int j = 0; j < kGenV; ++j) wr[j] = wi[j] = 0.f;
  // groups of kGenQ rows: the rows' phase loads are issued together, then
  // the rows are combined and stored
  constexpr int kGenQ = 4;
  static_assert(kGenRows % kGenQ == 0, "row groups");
  for (int r0 = 0; r0 < kGenRows; r0 += kGenQ) {
    int prow[kGenQ], tab[kGenQ];
#pragma unroll
    for (int q = 0; q < kGenQ; ++q) {
      const int m = m0 + r0 + q;
      if (UNEVEN) {  // (particle, translation, phase table) from the row table
        const int4 rw = m < Mrows ? rows[m] : make_int4(0, 0, 0, 0);
        prow[q] = rw.x;
        tab[q] = rw.z;
      } else {
        prow[q] = p;
        tab[q] = t;
        if (++t == T) {
          t = 0;
          ++p;
        }
      }
    }
    float4 f[kGenQ][2];
#pragma unroll
    for (int q = 0; q < kGenQ; ++q) {
      if (m0 + r0 + q < Mrows) {
        const float4* pp = reinterpret_cast<const float4*>(ph + (size_t)tab[q] * Kh + kp0);
        f[q][0] = pp[0];
        f[q][1] = pp[1];
      } else {
        f[q][0] = f[q][1] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
#pragma unroll
    for (int q = 0; q < kGenQ; ++q) {
      const int m = m0 + r0 + q;
      float ar[kGenV], ai[kGenV];
#pragma unroll
      for (int j = 0; j < kGenV; ++j) ar[j] = ai[j] = 0.f;
      if (m < Mrows) {
        if (prow[q] != cur_p) {
          const int pq = prow[q];
          const float sc = inv_sa ? __frcp_rn(inv_sa[pq]) : 1.f;  // FP16 forms: exact power-of-two scale
#pragma unroll
          for (int j = 0; j < kGenV; ++j) {
            float w = 0.f, xr = 0.f, xi = 0.f;
            if (pix[j] >= 0) {
              if (parts) {
                const PartDev& pd = parts[pq];
                w = pd.corr[pix[j]] / 2;
                xr = pd.re[pix[j]];
                xi = pd.im[pix[j]];
              } else {
                const long long at = (long long)pq * stride + pix[j];
                w = corr[at] / 2;
                xr = re[at];
                xi = im[at];
              }
            }
            wr[j] = w * xr;
            wi[j] = w * xi;
            if (inv_sa) {
              wr[j] *= sc;
              wi[j] *= sc;
            }
          }
          cur_p = pq;
        }
        const float pr[kGenV] = {f[q][0].x, f[q][0].z, f[q][1].x, f[q][1].z};
        const float pi[kGenV] = {f[q][0].y, f[q][0].w, f[q][1].y, f[q][1].w};
#pragma unroll
        for (int j = 0; j < kGenV; ++j) {
          ar[j] = __fmaf_rn(wr[j], pr[j], -__fmul_rn(wi[j], pi[j]));
          ai[j] = __fmaf_rn(wr[j], pi[j], __fmul_rn(wi[j], pr[j]));
        }
      }
      store_split4<PREC>(ahi, alo, (size_t)m * Kh + kp0, ar, ai);
    }
  }
}

template <int PREC, int ROWB, int BN>
struct GemmCfg {
  static constexpr bool kTf32 = (PREC == B200D2_PREC_TF32 || PREC == B200D2_PREC_TF32X3);
  static constexpr bool kScaled = (PREC == B200D2_PREC_FP16 || PREC == B200D2_PREC_FP16X3);
  static constexpr int kElem = kTf32 ? 4 : 2;
  static constexpr int kRowB = ROWB;
  static constexpr int kBK = ROWB / kElem;       // elements per k-block row
  static constexpr int kKStep = kTf32 ? 8 : 16;  // K of one tcgen05.mma (32 bytes)
  static constexpr int kTerms = (PREC == B200D2_PREC_TF32 || PREC == B200D2_PREC_FP16) ? 1 : 3;
  // operand format of the instruction descriptor: TF32 = 2 (kind::tf32),
  // BF16 = 1 and F16 = 0 (kind::f16)
  static constexpr uint32_t kFmt = kTf32 ? 2u : (PREC == B200D2_PREC_BF16X3 ? 1u : 0u);
  static constexpr int kPlanes = kTerms == 3 ? 2 : 1;
  static constexpr int kBM = 128, kBN = BN;
  static constexpr int kTmemCols = 2 * BN;  // a power of two >= 32
  static constexpr int kATile = kBM * ROWB;
  static constexpr int kBTile = kBN * ROWB;
  static constexpr int kStageBytes = kPlanes * (kATile + kBTile);
  static constexpr int kStages = (200 * 1024) / kStageBytes < 8 ? (200 * 1024) / kStageBytes : 8;
  static constexpr uint32_t kIdesc = sm100::idesc_f32acc(kFmt, kBM, kBN);
  static constexpr int kBarBytes = 256;
  static constexpr int kSmem = kStages * kStageBytes + kBarBytes + 1024;
  static_assert(kStages >= 2, "at least two pipeline stages");
  static_assert(3 * kStages * 8 + 5 * 8 + 8 <= kBarBytes, "barrier area");
  static_assert(BN == 128 || BN == 256, "tile width");
};

struct GemmArgs {
  int Mrows, Mtiles, Ntiles, O, T, KB, accumulate;
  int group_m;  // uniform batches: 0 = m-major tile order, else groups of group_m m-tiles, n-major inside
  int split;    // k-splits per tile (>= 1)
  float* out;
  const double* na;
  const float2* na_hl;  // nA = hi + lo (double-float)
  int combine64;        // 1: FP64 combine; 0: double-float combine
  int cc;               // 1: CC score k c (na holds k), 0: diff2 nA - 2c
  unsigned long long* keys;
  uint32_t* status;
  const float* inv_sa;  // FP16 forms: [P] 1 / particle scale
  const float* inv_sb;  // FP16 forms: [Opad] 1 / orientation scale
  float* part;          // split > 1: [tiles * split][BN][128] FP32 partial sums
  unsigned* cnt;        // split > 1: [tiles][8] arrivals per (tile, column half, TMEM lane quadrant)
  Layout L;  // uneven batch tables (all null for a uniform batch)
  // limit (ns) of the single-CTA kernel's pipeline waits (stage ring and
  // accumulator hand-over); its drain waits keep kWaitLimitNs
  unsigned long long wait_ns;
  // operand generation in the contraction (GEN kernels)
  const float2* wx;    // [P][Kh] weighted images of the listed pixels
  const int2* xy;      // [K_c] listed pixel coordinates
  const float2* ph;    // [tables][Kh] phase products (when the shared rows do not fit)
  const int2* cxy;     // [tables] rows of the compact phase tables
  const int* thdr;     // {rows x, rows y, extent, fits}
  const float2* exc;   // compact e^{i x tx} rows
  const float2* eyc;   // compact e^{i y ty} rows
  int Kh, K_c;
  int P;               // particles (row P of wx is all zero)
};

// (m0, n0) of the tile-th tile: the work list of an uneven batch, or the
// dense order of a uniform one.
__device__ __forceinline__ void tile_origin(const GemmArgs& g, int tile, int bm, int bn, int& m0, int& n0) {
  if (g.L.tiles) {
    const int2 mn = g.L.tiles[tile];
    m0 = mn.x * bm;
    n0 = mn.y * bn;
  } else if (g.group_m > 0) {
    // groups of group_m m-tiles whose A rows stay in L2 while every n-tile
    // (B rows) streams past them once per group
    const int per_group = g.group_m * g.Ntiles;
    const int grp = tile / per_group, rem = tile - grp * per_group;
    const int gm0 = grp * g.group_m, gsz = min(g.group_m, g.Mtiles - gm0);
    m0 = (gm0 + rem % gsz) * bm;
    n0 = (rem / gsz) * bn;
  } else {
    m0 = (tile / g.Ntiles) * bm;
    n0 = (tile % g.Ntiles) * bn;
  }
}

// k-blocks [kb0, kb1) of split s of a tile
__device__ __forceinline__ void split_range(const GemmArgs& g, int s, int& kb0, int& kb1) {
  kb0 = (int)(((long long)g.KB * s) / g.split);
  kb1 = (int)(((long long)g.KB * (s + 1)) / g.split);
}

__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float from_ordered(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s

// Pipeline-wait limit of the single-CTA contraction, set by
// b200d2_set_wait_limit_ns for tests of the give-up path (0: kWaitLimitNs).
static std::atomic<unsigned long long> g_wait_ns{0};

// Epilogue warps of the contraction kernels: two per TMEM lane quadrant, each
// draining half of the accumulator's columns.
constexpr int kEpiWarps = 8;
constexpr int kGemmThreads = 64 + 32 * kEpiWarps;  // TMA warp, MMA warp, epilogue warps

// One row of a tile in the epilogue: where its diff2 values go and what they
// combine with.
struct EpiRow {
  float* out_row;          // diff2 of (particle, translation) at orientation list index 0
  const double* na_row;    // FP64 nA of the particle, per orientation
  const float2* nh_row;    // the same as hi + lo floats
  const int* inv;          // orientation -> list index of the particle (uneven batches), or null
  int Tp, t;               // translations of the particle, this row's translation
  double m2s;              // -2 / (particle scale of the FP16 forms), else -2
  float m2f;
};

// Combine one accumulator value c of orientation o: diff2 = nA - 2c, stored,
// with the running minimum (value and orientation list index).  nA carries 48
// bits (FP64 norms); the default double-float form rounds nA_hi - 2c once
// (FMA) and adds nA_lo, within 2 ulp of the FP64 combine rounded to FP32, at
// about a tenth of its cost on this GPU.
//
// EpiCol: the per-column operands of the combine, loaded ahead of it: the
// local column (-1: not stored), nA in FP64 or as a double-float, and the
// FP16 orientation scale.
struct EpiCol {
  int lo;
  double na;
  float2 nh;
  float isb;
};

template <bool SCALED>
__device__ __forceinline__ EpiCol epi_col(const GemmArgs& g, const EpiRow& x, int o) {
  EpiCol k;
  k.lo = (o < g.O) ? (x.inv ? x.inv[o] : o) : -1;
  k.na = 0.0;
  k.nh = make_float2(0.f, 0.f);
  k.isb = 1.f;
  if (k.lo >= 0) {
    if (g.combine64)
      k.na = x.na_row[o];
    else
      k.nh = x.nh_row[o];
    if (SCALED) k.isb = g.inv_sb[o];
  }
  return k;
}

template <bool SCALED>
__device__ __forceinline__ void epi_combine_col(const GemmArgs& g, const EpiRow& x, const EpiCol& k, float c,
                                                float& best, int& best_lo) {
  const int lo = k.lo;
  if (lo < 0) return;
  float f;
  if (g.combine64) {
    double cr = (double)c;
    if (SCALED) cr *= (double)k.isb;
    // CC: k * c with the scales undone (-m2s/2 is the particle's, exact)
    f = g.cc ? (float)(k.na * (cr * (-0.5 * x.m2s))) : (float)fma(x.m2s, cr, k.na);
  } else {
    const float2 nh = k.nh;
    const float sc = SCALED ? x.m2f * k.isb : x.m2f;  // product of powers of two: exact
    f = g.cc ? __fmul_rn(nh.x, c * (-0.5f * sc)) : __fadd_rn(__fmaf_rn(sc, c, nh.x), nh.y);
  }
  float* dst = x.out_row + (size_t)lo * x.Tp;
  if (g.accumulate) f += __ldcs(dst);
  __stcs(dst, f);  // streamed: the output must not evict the operands from L2
  if (f < best) {
    best = f;
    best_lo = lo;
  }
}

template <bool SCALED>
__device__ __forceinline__ void epi_combine(const GemmArgs& g, const EpiRow& x, int o, float c, float& best,
                                            int& best_lo) {
  epi_combine_col<SCALED>(g, x, epi_col<SCALED>(g, x, o), c, best, best_lo);
}

// Drain NCH 32-column chunks of one TMEM lane quadrant starting at `taddr`
// (orientations from o0) into diff2.  `fast`: a uniform batch whose columns
// all exist, overwritten, double-float combine (no per-element branches).
template <bool SCALED, int NCH>
__device__ __forceinline__ void epi_drain(const GemmArgs& g, const EpiRow& x, uint32_t taddr, int o0, bool vrow,
                                          bool fast, float& best, int& best_lo) {
  uint32_t ra[32];
  auto use = [&](const uint32_t (&r)[32], int oc) {
    if (!vrow) return;
    if (fast) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int o = oc + j;
        const float2 nh = x.nh_row[o];
        const float sc = SCALED ? x.m2f * g.inv_sb[o] : x.m2f;
        const float c = __uint_as_float(r[j]);
        const float f = g.cc ? __fmul_rn(nh.x, c * (-0.5f * sc)) : __fadd_rn(__fmaf_rn(sc, c, nh.x), nh.y);
        __stcs(x.out_row + (size_t)o * x.Tp, f);
        if (f < best) {
          best = f;
          best_lo = o;
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) epi_combine<SCALED>(g, x, oc + j, __uint_as_float(r[j]), best, best_lo);
    }
  };
#pragma unroll 1
  for (int c = 0; c < NCH; ++c) {
    __syncwarp();
    sm100::tmem_ld_32x32b_x32(taddr + (uint32_t)(c * 32), ra);
    sm100::tmem_ld_wait_regs(ra);
    use(ra, o0 + c * 32);
  }
}

// ------------------------------------------------------------ A in shared memory
// Operand generation inside the contraction: kGenWarps extra warps write each
// k-block of A (128 rows of the weighted, phase-shifted images, split into
// hi/lo planes) straight into the stage ring, in the layout TMA would have
// written (K-major rows of ROWB bytes, 128- or 64-byte swizzle), so A never
// goes through global memory.  Element (row m = (p, t), listed pixel k):
//   a = wx[p][k] * ph,  ph = ex[x(k)] * ey[y(k)] of translation t
// with the products rounded exactly as tc_phase2d_kernel and tc_gen_a_kernel
// round them: the operands are bit-identical to the materialised ones.  The
// deduplicated phase rows (tc_phase_compact_kernel) sit in shared memory; when
// they do not fit, ph is read from the (table, pixel) products in global
// memory instead (same values).
// The generating kernels have 4 epilogue warps (one per TMEM lane quadrant,
// all columns; with the double-float combine they need a few thousand cycles
// of a tile's tens of thousands) and 8 generator warps in two groups that
// take alternate k-blocks: 448 threads, the most that 128 registers per
// thread allow (four warps per SM sub-partition).
constexpr int kEpiWarpsGen = 4;
constexpr int kGenWarps = 8;
constexpr int kGenFirstWarp = 2 + kEpiWarpsGen;
constexpr int kGemmThreadsGen = 64 + 32 * (kEpiWarpsGen + kGenWarps);
constexpr int kGenTabEntries = 1920;                   // float2 entries of the shared phase rows
constexpr int kGenTabBytes = kGenTabEntries * 8;       // 15 KB
// per generator warp: a k-block's pixel coordinates and the weighted images
// of up to 8 particle runs (32 pixels each, 33 entries apart)
constexpr int kGenSlotBytes = kGenWarps * (32 * 8 + 8 * 33 * 8);
constexpr int kSmemLimit = 227 * 1024;

// Byte offset of byte b of row R in a K-major tile of ROWB-byte rows written
// with TMA's 128-byte (ROWB 128) or 64-byte (ROWB 64) swizzle: the 16-byte
// chunk index is XORed with address bits 7-9 (7-8); tiles are 1024-byte aligned.
template <int ROWB>
__device__ __forceinline__ uint32_t swz_off(int R, int b) {
  if constexpr (ROWB == 128)
    return (uint32_t)(R * 128 + ((((b >> 4) ^ (R & 7)) << 4) | (b & 15)));
  else
    return (uint32_t)(R * 64 + ((((b >> 4) ^ ((R >> 1) & 3)) << 4) | (b & 15)));
}

// Split of the element pair (re, im) of one pixel into the hi and lo words of
// the 2-byte forms (the same values as store_split): bf16x2 / half2 bits.
template <int PREC>
__device__ __forceinline__ void split_words(float re, float im, uint32_t& hi, uint32_t& lo) {
  if constexpr (PREC == B200D2_PREC_BF16X3) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  } else if constexpr (PREC == B200D2_PREC_FP16X3) {
    const __half2 h = __floats2half2_rn(re, im);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(re - hf.x, im - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  } else {  // FP16 (one plane)
    const __half2 h = __floats2half2_rn(re, im);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = 0u;
  }
}

// (the phase rows are written once, before the named barrier that precedes
// every read, so the loads need no ordering against other memory operations)
__device__ __forceinline__ float2 lds_f2(uint32_t addr) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

// (no memory clobber: nothing this thread loads aliases the operand tiles, and
// volatile asm keeps the stores ordered with the barrier waits and the proxy
// fence around them)
__device__ __forceinline__ void sts_u4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d));
}

// 8-byte asynchronous copy global -> shared (zero-filled when !pred; the
// source is then not read)
__device__ __forceinline__ void cp_async8_u32(uint32_t smem, const void* gmem, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem), "l"(gmem), "r"(pred ? 8 : 0) : "memory");
}

// One generator warp.  The generator warps form two groups of four, which
// take the k-blocks of this CTA in turns (group gw / 4 the k-blocks of that
// parity in the CTA's sequence), so consecutive stages are written at the
// same time; within a group warp gw owns rows (gw % 4) * 32 .. + 31 of the
// CTA's 128-row tile.  Lane i keeps its row's particle, translation and
// phase rows in registers for the whole tile and writes the row's k-block a
// 16-byte chunk (VPC pixels) at a time: within a warp the chunks of eight
// consecutive rows fall on distinct banks under the swizzle, so the stores
// are conflict-free.  A row's particle is one of few: a particle's rows are
// contiguous, so the warp's 32 rows form runs.  The k-block's pixel
// coordinates and the weighted images of the first kGenRuns runs are copied
// into the warp's shared slots with cp.async as soon as the warp has handed
// over its previous k-block (they land while the other group writes), so the
// element loop reads shared memory only; rows of later runs (batches with
// fewer than about four translations per particle) read their weighted image
// from global memory.
constexpr int kGenRuns = 8;
template <int PREC, int ROWB>
struct GenWarp {
  static constexpr bool kTf32 = (PREC == B200D2_PREC_TF32 || PREC == B200D2_PREC_TF32X3);
  static constexpr int kElem = kTf32 ? 4 : 2;
  static constexpr int PPR = ROWB / (2 * kElem);  // complex pixels per row of a k-block
  static constexpr int VPC = 16 / (2 * kElem);    // pixels per 16-byte chunk
  static constexpr int NCH = ROWB / 16;           // chunks per row
  static constexpr int RPW = 32 / PPR;            // runs staged per warp-wide copy
  static constexpr int kCoordSlot = 32 * 8;       // bytes of a warp's coordinate slots
  // runs PPR + 1 entries apart (odd word-pair stride): rows of different runs
  // read distinct banks
  static constexpr int kRunStride = PPR + 1;
  static constexpr int kWSlot = kGenRuns * 33 * 8;
  const GemmArgs& g;
  int lane;
  uint32_t s_ex, s_ey;  // shared addresses of the phase rows (when fits)
  uint32_t s_coord;     // this warp's coordinate slots [PPR] int2
  uint32_t s_w;         // this warp's weighted-image slots [kGenRuns][PPR] float2
  int ext, fits;
  // this lane's row
  bool valid;
  uint32_t ex_row, ey_row;  // shared addresses of the row's e^{i x tx} and e^{i y ty} rows
  const float2* wx_row;     // weighted image of the row's particle (global)
  const float2* ph_row;     // (translation, pixel) products of the row's table (when the rows do not fit)
  int R;                    // row within the CTA's tile
  int run, nruns;           // this row's run and the runs staged in shared memory
  int run_p;                // lane r < runs: particle row of run r

  __device__ __forceinline__ GenWarp(const GemmArgs& g_, int gw, int lane_, uint32_t s_ex_, uint32_t s_ey_,
                                     uint32_t s_slots, int ext_, int fits_)
      : g(g_), lane(lane_), s_ex(s_ex_), s_ey(s_ey_), ext(ext_), fits(fits_) {
    R = (gw % 4) * 32 + lane;
    s_coord = s_slots + (uint32_t)gw * kCoordSlot;
    s_w = s_slots + (uint32_t)kGenWarps * kCoordSlot + (uint32_t)gw * kWSlot;
  }

  __device__ __forceinline__ void begin_tile(int m0) {
    const int m = m0 + R;
    valid = m < g.Mrows;
    int p = 0, t = 0;
    if (valid) {
      if (g.L.rows) {
        const int4 rw = g.L.rows[m];
        p = rw.x;
        t = rw.z;
      } else {
        p = m / g.T;
        t = m - p * g.T;
      }
    }
    // rows past the batch read the all-zero row after the last particle, so
    // their elements come out zero without a branch
    const int pe = valid ? p : g.P;
    wx_row = g.wx + (size_t)pe * g.Kh;
    ph_row = g.ph + (size_t)t * g.Kh;
    int2 cx = make_int2(0, 0);
    if (fits && valid) cx = g.cxy[t];
    ex_row = s_ex + (uint32_t)(cx.x * (ext + 1)) * 8u;
    ey_row = s_ey + (uint32_t)(cx.y * (2 * ext + 1) + ext) * 8u;
    // runs of equal particle rows
    const int prev = __shfl_up_sync(0xffffffffu, pe, 1);
    const unsigned runs = __ballot_sync(0xffffffffu, lane == 0 || pe != prev);
    run = __popc(runs & ((2u << lane) - 1u)) - 1;
    const int n = __popc(runs);
    nruns = n < kGenRuns ? n : kGenRuns;
    run_p = __shfl_sync(0xffffffffu, pe, lane < n ? (int)__fns(runs, 0, lane + 1) : 0);
  }

  // copy k-block kb's coordinates and the staged runs' weighted images into
  // the slots (one cp.async group; the slots' previous contents have been read)
  __device__ __forceinline__ void stage(int kb) {
    const int k0 = kb * PPR;
    if (lane < PPR) {
      const int kp = k0 + lane;
      const bool ok = kp < g.K_c;
      cp_async8_u32(s_coord + (uint32_t)lane * 8u, ok ? (const void*)(g.xy + kp) : (const void*)g.xy, ok);
    }
    const int px = lane % PPR;
#pragma unroll
    for (int i = 0; i < (kGenRuns + RPW - 1) / RPW; ++i) {
      const int r = i * RPW + lane / PPR;
      const int pr = __shfl_sync(0xffffffffu, run_p, r < 32 ? r : 31);
      if (r < nruns)
        cp_async8_u32(s_w + (uint32_t)(r * kRunStride + px) * 8u, g.wx + (size_t)pr * g.Kh + k0 + px, true);
    }
    cp_async_commit();
  }

  // element (re, im) of this row at pixel j (w_sh: the row's staged weighted
  // image in shared memory, or wk the global one; pk: phase products)
  template <bool FITS, bool SHARED_W>
  __device__ __forceinline__ float2 element(uint32_t w_sh, const float2* wk, const float2* pk, int j) {
    float pr, pi;
    if constexpr (FITS) {
      int xs, ys;
      asm("ld.shared.v2.b32 {%0, %1}, [%2];" : "=r"(xs), "=r"(ys) : "r"(s_coord + 8u * (uint32_t)j));
      const float2 fx = lds_f2(ex_row + (uint32_t)xs * 8u);
      const float2 fy = lds_f2(ey_row + (uint32_t)ys * 8u);
      pr = __fmaf_rn(fx.x, fy.x, -__fmul_rn(fx.y, fy.y));
      pi = __fmaf_rn(fx.x, fy.y, __fmul_rn(fx.y, fy.x));
    } else {
      const float2 v = pk[j];
      pr = v.x;
      pi = v.y;
    }
    const float2 w = SHARED_W ? lds_f2(w_sh + 8u * (uint32_t)j) : wk[j];
    return make_float2(__fmaf_rn(w.x, pr, -__fmul_rn(w.y, pi)), __fmaf_rn(w.x, pi, __fmul_rn(w.y, pr)));
  }

  // write k-block kb (staged in the slots) into the tiles at shared addresses
  // hi / lo (FITS: the phase rows are in shared memory)
  template <bool FITS, bool SHARED_W>
  __device__ __forceinline__ void write_rows(int kb, uint32_t hi, uint32_t lo) {
    const uint32_t w_sh = s_w + (uint32_t)((run < kGenRuns ? run : 0) * kRunStride) * 8u;
    const float2* wk = wx_row + kb * PPR;
    const float2* pk = ph_row + kb * PPR;
    // half a row's chunks in flight (4 for 128-byte rows, 2 for 64-byte ones):
    // enough independent work to cover the loads' and the arithmetic chains'
    // latency within the 128-register budget
    constexpr int kUnroll = NCH / 2;
#pragma unroll kUnroll
    for (int q = 0; q < NCH; ++q) {
      const uint32_t off = swz_off<ROWB>(R, q * 16);
      if constexpr (kTf32) {
        float v[4];
#pragma unroll
        for (int j = 0; j < VPC; ++j) {
          const float2 a = element<FITS, SHARED_W>(w_sh, wk, pk, q * VPC + j);
          v[2 * j] = a.x;
          v[2 * j + 1] = a.y;
        }
        float h[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) h[e] = tf32_round(v[e]);
        sts_u4(hi + off, __float_as_uint(h[0]), __float_as_uint(h[1]), __float_as_uint(h[2]), __float_as_uint(h[3]));
        if constexpr (PREC == B200D2_PREC_TF32X3)
          sts_u4(lo + off, __float_as_uint(tf32_round(v[0] - h[0])), __float_as_uint(tf32_round(v[1] - h[1])),
                 __float_as_uint(tf32_round(v[2] - h[2])), __float_as_uint(tf32_round(v[3] - h[3])));
      } else {
        uint32_t h[4], l[4];
#pragma unroll
        for (int j = 0; j < VPC; ++j) {
          const float2 a = element<FITS, SHARED_W>(w_sh, wk, pk, q * VPC + j);
          split_words<PREC>(a.x, a.y, h[j], l[j]);
        }
        sts_u4(hi + off, h[0], h[1], h[2], h[3]);
        if constexpr (PREC != B200D2_PREC_FP16) sts_u4(lo + off, l[0], l[1], l[2], l[3]);
      }
    }
  }

  // k-block kb, its slots complete (cp.async.wait_group + __syncwarp by the caller)
  __device__ __forceinline__ void write(int kb, uint32_t hi, uint32_t lo) {
    const bool all_shared = __all_sync(0xffffffffu, run < kGenRuns);
    if (fits) {
      if (all_shared)
        write_rows<true, true>(kb, hi, lo);
      else
        write_rows<true, false>(kb, hi, lo);
    } else {
      if (all_shared)
        write_rows<false, true>(kb, hi, lo);
      else
        write_rows<false, false>(kb, hi, lo);
    }
  }
};

// Shared phase rows: copied from the compact tables by the generator warps
// (a named barrier over those warps alone) when they fit; s_ex / s_ey are
// their shared addresses.
__device__ __forceinline__ void gen_load_tables(const GemmArgs& g, float2* s_tab, int& ext, int& fits,
                                                uint32_t& s_ex, uint32_t& s_ey) {
  const int nrx = g.thdr[0], nry = g.thdr[1];
  ext = g.thdr[2];
  fits = g.thdr[3];
  const int ew = ext + 1, yw = 2 * ext + 1;
  s_ex = sm100::smem_u32(s_tab);
  s_ey = s_ex + (uint32_t)(nrx * ew) * 8u;
  if (fits) {
    const int tid = threadIdx.x - 32 * kGenFirstWarp;
    for (int i = tid; i < nrx * ew; i += 32 * kGenWarps) s_tab[i] = g.exc[i];
    for (int i = tid; i < nry * yw; i += 32 * kGenWarps) s_tab[nrx * ew + i] = g.eyc[i];
  }
  asm volatile("bar.sync 1, %0;" ::"n"(32 * kGenWarps) : "memory");
}

// Dynamic shared memory of a contraction configuration: the stage ring, the
// barriers, 1024 bytes of alignment slack and, when the kernel generates A,
// the shared phase rows and the generator warps' slots.
template <class C, bool GEN>
constexpr int gemm_smem_bytes() {
  return C::kStages * C::kStageBytes + C::kBarBytes + 1024 + (GEN ? kGenTabBytes + kGenSlotBytes : 0);
}

// Persistent contraction.  Work items are (tile, k-split) pairs, item =
// tile * split + s, handed out round-robin over the grid.  Warp 0 streams the
// operand k-blocks with TMA into a ring of shared-memory stages, warp 1 issues
// the tcgen05 MMAs into one of two TMEM accumulators, warps 2-5 (one per TMEM
// lane quadrant) drain the other accumulator.  With split == 1 the epilogue
// combines directly; with split > 1 each split stores its FP32 partial and the
// last split to arrive for a (tile, quadrant) adds all partials in split order
// (FP64) and combines, so the result does not depend on arrival order.
template <int PREC, int ROWB, int BN, bool GEN>
__global__ void __launch_bounds__(GEN ? kGemmThreadsGen : kGemmThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
                   const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo,
                   const __grid_constant__ GemmArgs g) {
  using C = GemmCfg<PREC, ROWB, BN>;
  static_assert(gemm_smem_bytes<C, GEN>() <= kSmemLimit, "shared memory");
  constexpr int EPI = GEN ? kEpiWarpsGen : kEpiWarps;  // epilogue warps
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::kStages * C::kStageBytes);  // TMA bytes
  uint64_t* empty = full + C::kStages;
  uint64_t* gfull = empty + C::kStages;  // GEN: generator warps' arrivals
  uint64_t* accf = gfull + C::kStages;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile uint32_t* s_abort = tmem_slot + 1;
  // GEN: shared phase rows
  float2* s_tab = reinterpret_cast<float2*>(smem + C::kStages * C::kStageBytes + C::kBarBytes);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; ++s) {
      sm100::mbar_init(&full[s], 1);             // the TMA warp's arrival and its bytes
      sm100::mbar_init(&empty[s], 1);
      sm100::mbar_init(&gfull[s], kGenWarps / 2);  // GEN: one arrival per warp of the group writing it
    }
    for (int b = 0; b < 2; ++b) {
      sm100::mbar_init(&accf[b], 1);
      sm100::mbar_init(&acce[b], 32 * EPI);
    }
    sm100::mbar_init(drain, 1);
    *s_abort = 0;
    sm100::fence_barrier_init();
    sm100::fence_proxy_async_smem();
  }
  if (warp == 0 && lane == 0) {
    if (!GEN) sm100::prefetch_tensormap(&mAhi);
    sm100::prefetch_tensormap(&mBhi);
    if (C::kPlanes == 2) {
      if (!GEN) sm100::prefetch_tensormap(&mAlo);
      sm100::prefetch_tensormap(&mBlo);
    }
  }
  if (warp == 1) {
    sm100::tmem_alloc(tmem_slot, C::kTmemCols);
    sm100::tmem_relinquish();
  }
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int num_tiles = g.L.tiles ? g.L.ntiles : g.Mtiles * g.Ntiles;
  const int num_items = num_tiles * g.split;

  auto raise_abort = [&]() {
    *s_abort = 1;
    atomicExch(g.status, (uint32_t)B200D2_ERR_TIMEOUT);
  };

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      // projections (B) are re-read by every m-tile: keep them in L2
      const uint64_t keep = sm100::policy_evict_last();
      uint32_t gk = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < num_items && ok; item += gridDim.x) {
        const int tile = item / g.split;
        int m0, n0, kb0, kb1;
        tile_origin(g, tile, C::kBM, C::kBN, m0, n0);
        split_range(g, item - tile * g.split, kb0, kb1);
        for (int kb = kb0; kb < kb1; ++kb, ++gk) {
          const int s = gk % C::kStages;
          const uint32_t u = gk / C::kStages;
          if (u > 0 && !sm100::mbar_wait_bounded(&empty[s], (u - 1) & 1, s_abort, g.wait_ns)) {
            raise_abort();
            ok = false;
            break;
          }
          sm100::mbar_arrive_expect_tx(&full[s], GEN ? C::kPlanes * C::kBTile : C::kStageBytes);
          uint8_t* st = smem + s * C::kStageBytes;
          const int kc = kb * C::kBK;
          if (!GEN) {
            sm100::tma_load_2d(st, &mAhi, &full[s], kc, m0);
            if (C::kPlanes == 2) sm100::tma_load_2d(st + C::kATile, &mAlo, &full[s], kc, m0);
          }
          uint8_t* sb = st + C::kPlanes * C::kATile;
          sm100::tma_load_2d_hint(sb, &mBhi, &full[s], kc, n0, keep);
          if (C::kPlanes == 2) sm100::tma_load_2d_hint(sb + C::kBTile, &mBlo, &full[s], kc, n0, keep);
        }
      }
      // let the copies in flight land before the CTA can exit (full[] counts
      // the TMA bytes alone, so this completes also after a give-up)
      const uint32_t issued = gk;
      for (uint32_t j = (issued > (uint32_t)C::kStages ? issued - C::kStages : 0); j < issued; ++j)
        sm100::mbar_wait_drain(&full[j % C::kStages], (j / C::kStages) & 1, kWaitLimitNs);
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t gk = 0;
      int i = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < num_items && ok; item += gridDim.x, ++i) {
        const int b = i & 1;
        const uint32_t v = (uint32_t)(i >> 1);
        if (v > 0 && !sm100::mbar_wait_bounded(&acce[b], (v - 1) & 1, s_abort, g.wait_ns)) {
          raise_abort();
          break;
        }
        sm100::tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * C::kBN);
        int kb0, kb1;
        split_range(g, item - (item / g.split) * g.split, kb0, kb1);
        for (int kb = kb0; kb < kb1; ++kb, ++gk) {
          const int s = gk % C::kStages;
          const uint32_t u = gk / C::kStages;
          if (!sm100::mbar_wait_bounded(&full[s], u & 1, s_abort, g.wait_ns) ||
              (GEN && !sm100::mbar_wait_bounded(&gfull[s], u & 1, s_abort, g.wait_ns))) {
            raise_abort();
            ok = false;
            break;
          }
          sm100::tc_fence_after();
          const uint32_t st = sm100::smem_u32(smem + s * C::kStageBytes);
          const uint32_t a_hi = st, a_lo = st + C::kATile;
          const uint32_t b_hi = st + C::kPlanes * C::kATile, b_lo = b_hi + C::kBTile;
#pragma unroll
          for (int ks = 0; ks < C::kBK / C::kKStep; ++ks) {
            const uint32_t koff = (uint32_t)(ks * C::kKStep * C::kElem);
            const uint64_t dah = sm100::desc_k_sw(a_hi + koff, C::kRowB);
            const uint64_t dbh = sm100::desc_k_sw(b_hi + koff, C::kRowB);
            const uint32_t acc = (kb > kb0 || ks > 0) ? 1u : 0u;
            sm100::mma<C::kTf32>(d, dah, dbh, C::kIdesc, acc);
            if (C::kTerms == 3) {
              sm100::mma<C::kTf32>(d, dah, sm100::desc_k_sw(b_lo + koff, C::kRowB), C::kIdesc, 1u);
              sm100::mma<C::kTf32>(d, sm100::desc_k_sw(a_lo + koff, C::kRowB), dbh, C::kIdesc, 1u);
            }
          }
          sm100::mma_commit(&empty[s]);
        }
        if (ok) sm100::mma_commit(&accf[b]);
      }
      // every MMA issued by this thread has retired once `drain` fires (the
      // tensor memory is released after it)
      sm100::mma_commit(drain);
      if (!sm100::mbar_wait_drain(drain, 0, kWaitLimitNs)) raise_abort();
    }
  } else if (GEN && warp >= kGenFirstWarp) {
    // ------------------------------------------------ A generators (warps 10..13)
    int ext, fits;
    uint32_t s_ex, s_ey;
    gen_load_tables(g, s_tab, ext, fits, s_ex, s_ey);
    const int gw = warp - kGenFirstWarp;
    GenWarp<PREC, ROWB> gen(g, gw, lane, s_ex, s_ey, sm100::smem_u32(s_tab) + kGenTabBytes, ext, fits);
    const uint32_t par = (uint32_t)(gw / 4);  // this warp's group takes the k-blocks gk with gk % 2 == par
    uint32_t gk = 0;
    bool ok = true;
    for (int item = blockIdx.x; item < num_items && ok; item += gridDim.x) {
      const int tile = item / g.split;
      int m0, n0, kb0, kb1;
      tile_origin(g, tile, C::kBM, C::kBN, m0, n0);
      split_range(g, item - tile * g.split, kb0, kb1);
      gen.begin_tile(m0);
      bool pending = false;  // the next own k-block is already staged
      for (int kb = kb0; kb < kb1; ++kb, ++gk) {
        if ((gk & 1u) != par) continue;
        if (!pending) gen.stage(kb);
        const int s = gk % C::kStages;
        const uint32_t u = gk / C::kStages;
        int w = 1;
        if (u > 0 && lane == 0) w = sm100::mbar_wait_bounded(&empty[s], (u - 1) & 1, s_abort, g.wait_ns) ? 1 : 0;
        w = __shfl_sync(0xffffffffu, w, 0);
        if (!w) {
          if (lane == 0) raise_abort();
          ok = false;
          break;
        }
        cp_async_wait<0>();  // this k-block's slots have landed
        __syncwarp();
        const uint32_t st = sm100::smem_u32(smem + s * C::kStageBytes);
        gen.write(kb, st, st + C::kATile);
        sm100::fence_proxy_async_smem();  // the tensor cores read these tiles through the async proxy
        __syncwarp();
        if (lane == 0) sm100::mbar_arrive(&gfull[s]);
        // the next own k-block of this tile lands while the other group writes
        pending = kb + 2 < kb1;
        if (pending) gen.stage(kb + 2);
      }
    }
    cp_async_wait<0>();  // no copy into shared memory outlives the loop
  } else {
    // ------------------------------------------------ epilogue (warps 2 .. 2 + EPI - 1)
    // warp w may read TMEM lanes 32 (w % 4) .. +31; with 8 epilogue warps
    // warps 2-5 drain the first half of the columns and warps 6-9 the second,
    // with 4 each warp drains all columns of its quadrant
    const int qd = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = qd * 32 + lane;
    constexpr int kCols = C::kBN / (EPI / 4);  // columns per epilogue warp
    int i = 0;
    for (int item = blockIdx.x; item < num_items; item += gridDim.x, ++i) {
      const int b = i & 1;
      const uint32_t v = (uint32_t)(i >> 1);
      int ok = 1;
      if (lane == 0) ok = sm100::mbar_wait_bounded(&accf[b], v & 1, s_abort, g.wait_ns) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) raise_abort();
        break;
      }
      sm100::tc_fence_after();
      const int tile = item / g.split;
      int m0, n0;
      tile_origin(g, tile, C::kBM, C::kBN, m0, n0);
      const int m = m0 + row;
      const bool vrow = m < g.Mrows;
      int p = 0;
      EpiRow x;
      x.t = 0;
      x.Tp = g.T;
      x.out_row = g.out;
      x.inv = nullptr;
      if (vrow) {
        if (g.L.rows) {
          const int4 rw = g.L.rows[m];
          p = rw.x;
          x.t = rw.y;
          const PartDev& pd = g.L.parts[p];
          x.Tp = pd.T;
          x.out_row = pd.out;
          x.inv = pd.inv;
        } else {
          p = m / g.T;
          x.t = m - p * g.T;
          x.out_row = g.out + (size_t)p * g.O * g.T;
        }
      }
      x.out_row += x.t;
      x.na_row = g.na + (size_t)p * g.O;
      x.nh_row = g.na_hl + (size_t)p * g.O;
      // FP16 forms: -2 / (particle scale); the orientation scale is per column
      x.m2s = C::kScaled ? -2.0 * (double)g.inv_sa[p] : -2.0;
      x.m2f = (float)x.m2s;  // a power of two: exact
      const int o0 = n0 + half * kCols;
      const bool fast = !x.inv && !g.accumulate && !g.combine64 && o0 + kCols <= g.O;
      float best = __int_as_float(0x7f800000);
      int best_lo = -1;
      bool mine = true;  // this warp's rows and columns are combined by this item
      const uint32_t taddr = tmem + (uint32_t)(b * C::kBN + half * kCols) + ((uint32_t)(qd * 32) << 16);
      if (g.split == 1) {
        epi_drain<C::kScaled, kCols / 32>(g, x, taddr, o0, vrow, fast, best, best_lo);
        sm100::tc_fence_before();
        sm100::mbar_arrive(&acce[b]);
      } else {
        // store this split's partial: [item][column][row], coalesced over rows
        float* part = g.part + (size_t)item * C::kBN * 128 + (size_t)(half * kCols) * 128 + row;
#pragma unroll 1
        for (int c = 0; c < kCols / 32; ++c) {
          uint32_t r[32];
          __syncwarp();
          sm100::tmem_ld_32x32b_x32(taddr + (uint32_t)(c * 32), r);
          sm100::tmem_ld_wait_regs(r);
#pragma unroll
          for (int j = 0; j < 32; ++j) part[(size_t)(c * 32 + j) * 128] = __uint_as_float(r[j]);
        }
        sm100::tc_fence_before();
        sm100::mbar_arrive(&acce[b]);
        __threadfence();
        __syncwarp();
        const int ci = tile * 8 + half * 4 + qd;  // arrivals per (tile, column half, lane quadrant)
        unsigned last = 0;
        if (lane == 0) last = atomicAdd(&g.cnt[ci], 1u) == (unsigned)(g.split - 1) ? 1u : 0u;
        last = __shfl_sync(0xffffffffu, last, 0);
        mine = last != 0;
        if (mine) {
          __threadfence();
          const float* base = g.part + (size_t)tile * g.split * C::kBN * 128 + row;
          if (vrow) {
            // the partials of kSumCols columns are loaded together (their
            // loads overlap), then added in split order in FP64
            constexpr int kSumCols = 4;
            static_assert(kCols % kSumCols == 0, "column chunks");
#pragma unroll 1
            for (int col0 = half * kCols; col0 < (half + 1) * kCols; col0 += kSumCols) {
              float v[kSumCols][kMaxSplit];
              EpiCol kc[kSumCols];
#pragma unroll
              for (int c = 0; c < kSumCols; ++c) {
                kc[c] = epi_col<C::kScaled>(g, x, n0 + col0 + c);
#pragma unroll
                for (int s2 = 0; s2 < kMaxSplit; ++s2)
                  v[c][s2] = s2 < g.split ? __ldcg(base + ((size_t)s2 * C::kBN + col0 + c) * 128) : 0.f;
              }
#pragma unroll
              for (int c = 0; c < kSumCols; ++c) {
                double acc = 0.0;
#pragma unroll
                for (int s2 = 0; s2 < kMaxSplit; ++s2)
                  if (s2 < g.split) acc += (double)v[c][s2];
                epi_combine_col<C::kScaled>(g, x, kc[c], (float)acc, best, best_lo);
              }
            }
          }
          __syncwarp();
          if (lane == 0) g.cnt[ci] = 0;  // ready for the next launch
        }
      }
      if (mine) {
        // Per-particle minimum across the warp's 32 rows: a particle's rows
        // are contiguous, so a segmented shuffle-down min leaves each run's
        // minimum in its first lane, which alone issues the atomic.
        unsigned long long key =
            (vrow && best_lo >= 0)
                ? (((unsigned long long)ordered_bits(best) << 32) | (uint32_t)(best_lo * x.Tp + x.t))
                : ~0ull;
        const int pk = vrow ? p : -1;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const unsigned long long ok2 = __shfl_down_sync(0xffffffffu, key, off);
          const int op = __shfl_down_sync(0xffffffffu, pk, off);
          if (lane + off < 32 && op == pk && ok2 < key) key = ok2;
        }
        const int prevp = __shfl_up_sync(0xffffffffu, pk, 1);
        if (pk >= 0 && (lane == 0 || prevp != pk) && key != ~0ull) atomicMin(&g.keys[pk], key);
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    sm100::tc_fence_after();
    sm100::tmem_dealloc(tmem, C::kTmemCols);
  }
}

// CTA-pair variant (cta_group::2): a cluster of two CTAs computes a 256 x 256
// tile.  Each CTA loads its 128 rows of A and its 128-row half of B into its
// own shared memory; the even CTA issues one M = 256, N = 256 MMA per k-step
// that reads both CTAs' tiles, and each CTA's TMEM receives its own 128 rows
// of the accumulator.  Per SM the operand stream from L2 and the tensor core's
// shared-memory reads are a third lower than with a 128 x 256 tile per CTA.
// No k-splits; uneven batches through a work list of 256-row m-tiles.
template <int PREC, int ROWB>
struct GemmCfgPair {
  using Base = GemmCfg<PREC, ROWB, 256>;
  static constexpr bool kTf32 = Base::kTf32;
  static constexpr bool kScaled = Base::kScaled;
  static constexpr int kElem = Base::kElem, kBK = Base::kBK, kKStep = Base::kKStep, kTerms = Base::kTerms;
  static constexpr int kPlanes = Base::kPlanes, kRowB = ROWB;
  static constexpr int kBM = 128;  // rows of A per CTA (256 per pair)
  static constexpr int kBNh = 128;  // rows of B per CTA (N = 256 per pair)
  static constexpr int kATile = kBM * ROWB, kBTile = kBNh * ROWB;
  static constexpr int kStageBytes = kPlanes * (kATile + kBTile);
  static constexpr int kStages = (200 * 1024) / kStageBytes < 8 ? (200 * 1024) / kStageBytes : 8;
  static constexpr uint32_t kIdesc = sm100::idesc_f32acc(Base::kFmt, 256, 256);
  static constexpr int kTmemCols = 512;
  static constexpr int kBarBytes = 256;
  static constexpr int kSmem = kStages * kStageBytes + kBarBytes + 1024;
  static_assert(kStages >= 2, "at least two pipeline stages");
  static_assert(3 * kStages * 8 + 5 * 8 + 8 <= kBarBytes, "barrier area");
};

template <int PREC, int ROWB, bool GEN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEN ? kGemmThreadsGen : kGemmThreads, 1)
    tc_gemm_pair_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
                        const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo,
                        const __grid_constant__ GemmArgs g) {
  using C = GemmCfgPair<PREC, ROWB>;
  static_assert(gemm_smem_bytes<C, GEN>() <= kSmemLimit, "shared memory");
  constexpr int EPI = GEN ? kEpiWarpsGen : kEpiWarps;  // epilogue warps
  constexpr int kCols = 256 / (EPI / 4);                // columns per epilogue warp
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::kStages * C::kStageBytes);  // TMA bytes
  uint64_t* empty = full + C::kStages;
  uint64_t* gfull = empty + C::kStages;  // GEN: generator warps' arrivals
  uint64_t* accf = gfull + C::kStages;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile uint32_t* s_abort = tmem_slot + 1;
  float2* s_tab = reinterpret_cast<float2*>(smem + C::kStages * C::kStageBytes + C::kBarBytes);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = sm100::cluster_ctarank();  // 0 issues the MMAs
  const bool lead = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; ++s) {
      sm100::mbar_init(&full[s], 1);                  // used in the even CTA: its own arrive + both CTAs' bytes
      sm100::mbar_init(&empty[s], 1);                 // one multicast commit per use
      sm100::mbar_init(&gfull[s], kGenWarps);         // GEN, even CTA: the writing group's warps of both CTAs
    }
    for (int b = 0; b < 2; ++b) {
      sm100::mbar_init(&accf[b], 1);
      sm100::mbar_init(&acce[b], 2 * 32 * EPI);  // even CTA: the epilogue threads of both CTAs
    }
    sm100::mbar_init(drain, 1);
    *s_abort = 0;
    sm100::fence_barrier_init();
    sm100::fence_proxy_async_smem();
  }
  if (warp == 0 && lane == 0) {
    if (!GEN) sm100::prefetch_tensormap(&mAhi);
    sm100::prefetch_tensormap(&mBhi);
    if (C::kPlanes == 2) {
      if (!GEN) sm100::prefetch_tensormap(&mAlo);
      sm100::prefetch_tensormap(&mBlo);
    }
  }
  if (warp == 1) {
    sm100::tmem_alloc_pair(tmem_slot, C::kTmemCols);
    sm100::tmem_relinquish_pair();
  }
  sm100::tc_fence_before();
  __syncthreads();
  sm100::cluster_sync();  // both CTAs' barriers initialised before any remote use
  sm100::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int num_tiles = g.L.tiles ? g.L.ntiles : g.Mtiles * g.Ntiles;
  const int cl = blockIdx.x >> 1, ncl = gridDim.x >> 1;
  const uint32_t full0 = sm100::map_to_rank(full, 0);  // the even CTA's full[0]
  const uint32_t gfull0 = sm100::map_to_rank(gfull, 0);
  const uint32_t acce0 = sm100::map_to_rank(acce, 0);

  auto raise_abort = [&]() {
    *s_abort = 1;
    atomicExch(g.status, (uint32_t)B200D2_ERR_TIMEOUT);
  };

  if (warp == 0) {
    // ------------------------------------------------ TMA producer (both CTAs)
    if (lane == 0) {
      const uint64_t keep = sm100::policy_evict_last();  // B is re-read by every m-tile
      uint32_t gk = 0;
      bool ok = true;
      for (int tile = cl; tile < num_tiles && ok; tile += ncl) {
        int m0, n0;
        tile_origin(g, tile, 256, 256, m0, n0);
        for (int kb = 0; kb < g.KB; ++kb, ++gk) {
          const int s = gk % C::kStages;
          const uint32_t u = gk / C::kStages;
          if (u > 0 && !sm100::mbar_wait_bounded(&empty[s], (u - 1) & 1, s_abort, kWaitLimitNs)) {
            raise_abort();
            ok = false;
            break;
          }
          if (lead) sm100::mbar_arrive_expect_tx(&full[s], GEN ? 2 * C::kPlanes * C::kBTile : 2 * C::kStageBytes);
          uint8_t* st = smem + s * C::kStageBytes;
          const uint32_t fb = full0 + 8u * (uint32_t)s;
          const int kc = kb * C::kBK;
          if (!GEN) {
            sm100::tma_load_2d_pair(st, &mAhi, fb, kc, m0 + 128 * (int)rank);
            if (C::kPlanes == 2) sm100::tma_load_2d_pair(st + C::kATile, &mAlo, fb, kc, m0 + 128 * (int)rank);
          }
          uint8_t* sb = st + C::kPlanes * C::kATile;
          sm100::tma_load_2d_pair_hint(sb, &mBhi, fb, kc, n0 + 128 * (int)rank, keep);
          if (C::kPlanes == 2) sm100::tma_load_2d_pair_hint(sb + C::kBTile, &mBlo, fb, kc, n0 + 128 * (int)rank, keep);
        }
      }
      // the even CTA's full barriers count both CTAs' bytes: let every copy
      // in flight land before either CTA can leave (the final cluster
      // barrier holds the odd CTA until then)
      if (lead) {
        const uint32_t issued = gk;
        for (uint32_t j = (issued > (uint32_t)C::kStages ? issued - C::kStages : 0); j < issued; ++j)
          sm100::mbar_wait_drain(&full[j % C::kStages], (j / C::kStages) & 1, kWaitLimitNs);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer (even CTA)
    if (lead && lane == 0) {
      uint32_t gk = 0;
      int i = 0;
      bool ok = true;
      for (int tile = cl; tile < num_tiles && ok; tile += ncl, ++i) {
        const int b = i & 1;
        const uint32_t v = (uint32_t)(i >> 1);
        if (v > 0 && !sm100::mbar_wait_bounded(&acce[b], (v - 1) & 1, s_abort, kWaitLimitNs)) {
          raise_abort();
          break;
        }
        sm100::tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * 256);
        for (int kb = 0; kb < g.KB; ++kb, ++gk) {
          const int s = gk % C::kStages;
          const uint32_t u = gk / C::kStages;
          if (!sm100::mbar_wait_bounded(&full[s], u & 1, s_abort, kWaitLimitNs) ||
              (GEN && !sm100::mbar_wait_bounded(&gfull[s], u & 1, s_abort, kWaitLimitNs))) {
            raise_abort();
            ok = false;
            break;
          }
          sm100::tc_fence_after();
          const uint32_t st = sm100::smem_u32(smem + s * C::kStageBytes);
          const uint32_t a_hi = st, a_lo = st + C::kATile;
          const uint32_t b_hi = st + C::kPlanes * C::kATile, b_lo = b_hi + C::kBTile;
#pragma unroll
          for (int ks = 0; ks < C::kBK / C::kKStep; ++ks) {
            const uint32_t koff = (uint32_t)(ks * C::kKStep * C::kElem);
            const uint64_t dah = sm100::desc_k_sw(a_hi + koff, C::kRowB);
            const uint64_t dbh = sm100::desc_k_sw(b_hi + koff, C::kRowB);
            const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
            sm100::mma_pair<C::kTf32>(d, dah, dbh, C::kIdesc, acc);
            if (C::kTerms == 3) {
              sm100::mma_pair<C::kTf32>(d, dah, sm100::desc_k_sw(b_lo + koff, C::kRowB), C::kIdesc, 1u);
              sm100::mma_pair<C::kTf32>(d, sm100::desc_k_sw(a_lo + koff, C::kRowB), dbh, C::kIdesc, 1u);
            }
          }
          sm100::mma_commit_pair(&empty[s], (uint16_t)3);  // frees stage s in both CTAs
        }
        if (ok) sm100::mma_commit_pair(&accf[b], (uint16_t)3);
      }
      sm100::mma_commit_pair(drain, (uint16_t)1);
      if (!sm100::mbar_wait_drain(drain, 0, kWaitLimitNs)) raise_abort();
    }
  } else if (GEN && warp >= kGenFirstWarp) {
    // ------------------------------------------------ A generators (warps 10..13, both CTAs)
    // each CTA writes its own 128 rows; the stage completes on the even
    // CTA's barrier
    int ext, fits;
    uint32_t s_ex, s_ey;
    gen_load_tables(g, s_tab, ext, fits, s_ex, s_ey);
    const int gw = warp - kGenFirstWarp;
    GenWarp<PREC, ROWB> gen(g, gw, lane, s_ex, s_ey, sm100::smem_u32(s_tab) + kGenTabBytes, ext, fits);
    const uint32_t par = (uint32_t)(gw / 4);  // this warp's group takes the k-blocks gk with gk % 2 == par
    uint32_t gk = 0;
    bool ok = true;
    for (int tile = cl; tile < num_tiles && ok; tile += ncl) {
      int m0, n0;
      tile_origin(g, tile, 256, 256, m0, n0);
      gen.begin_tile(m0 + 128 * (int)rank);
      bool pending = false;  // the next own k-block is already staged
      for (int kb = 0; kb < g.KB; ++kb, ++gk) {
        if ((gk & 1u) != par) continue;
        if (!pending) gen.stage(kb);
        const int s = gk % C::kStages;
        const uint32_t u = gk / C::kStages;
        int w = 1;
        if (u > 0 && lane == 0) w = sm100::mbar_wait_bounded(&empty[s], (u - 1) & 1, s_abort, kWaitLimitNs) ? 1 : 0;
        w = __shfl_sync(0xffffffffu, w, 0);
        if (!w) {
          if (lane == 0) raise_abort();
          ok = false;
          break;
        }
        cp_async_wait<0>();  // this k-block's slots have landed
        __syncwarp();
        const uint32_t st = sm100::smem_u32(smem + s * C::kStageBytes);
        gen.write(kb, st, st + C::kATile);
        sm100::fence_proxy_async_smem();  // the tensor cores read these tiles through the async proxy
        __syncwarp();
        if (lane == 0) sm100::mbar_arrive_cluster(gfull0 + 8u * (uint32_t)s);
        // the next own k-block of this tile lands while the other group writes
        pending = kb + 2 < g.KB;
        if (pending) gen.stage(kb + 2);
      }
    }
    cp_async_wait<0>();  // no copy into shared memory outlives the loop
  } else {
    // ------------------------------------------------ epilogue (warps 2 .. 2 + EPI - 1, both CTAs)
    const int qd = warp & 3;            // TMEM lane quadrant this warp may access
    const int half = (warp - 2) >> 2;  // column half of the 256-wide tile (8 epilogue warps)
    const int row = qd * 32 + lane;
    int i = 0;
    for (int tile = cl; tile < num_tiles; tile += ncl, ++i) {
      const int b = i & 1;
      const uint32_t v = (uint32_t)(i >> 1);
      int ok = 1;
      if (lane == 0) ok = sm100::mbar_wait_bounded(&accf[b], v & 1, s_abort, kWaitLimitNs) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) raise_abort();
        break;
      }
      sm100::tc_fence_after();
      int m0, n0;
      tile_origin(g, tile, 256, 256, m0, n0);
      const int m = m0 + 128 * (int)rank + row;
      const bool vrow = m < g.Mrows;
      int p = 0;
      EpiRow x;
      x.t = 0;
      x.Tp = g.T;
      x.out_row = g.out;
      x.inv = nullptr;
      if (vrow) {
        if (g.L.rows) {
          const int4 rw = g.L.rows[m];
          p = rw.x;
          x.t = rw.y;
          const PartDev& pd = g.L.parts[p];
          x.Tp = pd.T;
          x.out_row = pd.out;
          x.inv = pd.inv;
        } else {
          p = m / g.T;
          x.t = m - p * g.T;
          x.out_row = g.out + (size_t)p * g.O * g.T;
        }
      }
      x.out_row += x.t;
      x.na_row = g.na + (size_t)p * g.O;
      x.nh_row = g.na_hl + (size_t)p * g.O;
      x.m2s = C::kScaled ? -2.0 * (double)g.inv_sa[p] : -2.0;
      x.m2f = (float)x.m2s;
      const int o0 = n0 + half * kCols;
      const bool fast = !x.inv && !g.accumulate && !g.combine64 && o0 + kCols <= g.O;
      float best = __int_as_float(0x7f800000);
      int best_lo = -1;
      epi_drain<C::kScaled, kCols / 32>(g, x, tmem + (uint32_t)(b * 256 + half * kCols) + ((uint32_t)(qd * 32) << 16),
                                        o0, vrow, fast, best, best_lo);
      sm100::tc_fence_before();
      sm100::mbar_arrive_cluster(acce0 + 8u * (uint32_t)b);  // the even CTA may reuse buffer b
      unsigned long long key =
          (vrow && best_lo >= 0)
              ? (((unsigned long long)ordered_bits(best) << 32) | (uint32_t)(best_lo * x.Tp + x.t))
              : ~0ull;
      const int pk = vrow ? p : -1;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long ok2 = __shfl_down_sync(0xffffffffu, key, off);
        const int op = __shfl_down_sync(0xffffffffu, pk, off);
        if (lane + off < 32 && op == pk && ok2 < key) key = ok2;
      }
      const int prevp = __shfl_up_sync(0xffffffffu, pk, 1);
      if (pk >= 0 && (lane == 0 || prevp != pk) && key != ~0ull) atomicMin(&g.keys[pk], key);
    }
  }
  __syncthreads();
  sm100::cluster_sync();  // no CTA leaves while its pair may still touch its memory
  if (warp == 1) {
    sm100::tc_fence_after();
    sm100::tmem_dealloc_pair(tmem, C::kTmemCols);
  }
}

// ------------------------------------------------------------------ stage 7
__global__ void tc_finalize_kernel(const unsigned long long* keys, int P, double* mn, long long* arg) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const unsigned long long k = keys[p];
  if (mn) mn[p] = (k == ~0ull) ? __longlong_as_double(0x7ff8000000000000LL) : (double)from_ordered((uint32_t)(k >> 32));
  if (arg) arg[p] = (k == ~0ull) ? -1 : (long long)(k & 0xffffffffull);
}

// ------------------------------------------------------------------ host side
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

static int make_map(CUtensorMap* m, void* base, int elem, int cols, int rows, int box_rows, int row_bytes,
                    bool fp16 = false) {
  auto enc = get_encode();
  if (!enc) return B200D2_ERR_CUDA;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * elem};
  const cuuint32_t box[2] = {(cuuint32_t)(row_bytes / elem), (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  const CUtensorMapDataType dt = elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : (fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16);
  CUresult r = enc(m, dt, 2,
                   base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? B200D2_OK : B200D2_ERR_CUDA;
}

static int num_sms() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// k-block row width used by the contraction (64 unless overridden by the
// B200D2_GEMM_ROW_BYTES environment variable: 64 or 128).
static int gemm_row_bytes() {
  static int rb = 0;
  if (rb == 0) {
    const char* e = getenv("B200D2_GEMM_ROW_BYTES");
    rb = (e && atoi(e) == 128) ? 128 : 64;
  }
  return rb;
}

// Contraction variant: k-block row width, tile width and k-splits per tile.
struct GemmVariant {
  int row_bytes = 0;  // 64 or 128; 0 = library default
  int bn = 0;         // orientations per tile: 256 or 128; 0 = library default (256)
  int split = 0;      // k-splits per tile; 0 = chosen from the tile count
  int pair = 0;       // 1: CTA-pair 256 x 256 tiles (uniform batches, no k-splits); 0: one CTA per tile
};

// Process-wide variant of the batch entry points (b200d2_set_gemm_variant);
// plans carry their own.
static std::atomic<int> g_var_rb{0}, g_var_bn{0}, g_var_split{0}, g_var_pair{0};
static std::atomic<int> g_combine64{0};  // b200d2_set_combine

// k-splits for `tiles` tiles of KB k-blocks: 1 when the tiles fill the GPU,
// else the largest power of two (<= cap) keeping two work items per SM at
// most and at least two k-blocks per split.
// A k-split stores every split's partial tile and has the last split add
// them (about 30 us at C1), so it pays only for long k-loops: each split
// keeps at least kSplitMinKB k-blocks (at C1, 28 k-blocks, splitting 4 ways
// took the contraction from 41 to 70 us).
constexpr int kSplitMinKB = 64;
static int auto_split(int tiles, int KB, int cap) {
  const int sms = num_sms();
  int sp = 1;
  if (tiles >= sms) return 1;
  while (sp * 2 <= cap && (long long)tiles * sp * 2 <= 2LL * sms && KB / (sp * 2) >= kSplitMinKB) sp *= 2;
  return sp;
}

// The operand-generation fields of the contraction's arguments.
static void set_gen_args(GemmArgs& a, const TcGeom& g, void* ws) {
  a.wx = ws_at<float2>(ws, g.off_wx);
  a.xy = ws_at<int2>(ws, g.off_xy);
  a.ph = ws_at<float2>(ws, g.off_ph);
  a.cxy = ws_at<int2>(ws, g.off_cxy);
  a.thdr = ws_at<int>(ws, g.off_thdr);
  a.exc = ws_at<float2>(ws, g.off_exc);
  a.eyc = ws_at<float2>(ws, g.off_eyc);
  a.Kh = g.Kpad / 2;
  a.K_c = g.K_c;
  a.P = g.P;
}

template <int PREC, int ROWB, int BN, bool GEN>
static int launch_gemm_v(const b200d2_batch& b, const TcGeom& g, void* ws, cudaStream_t s,
                         const UnevenTabs* U, int split) {
  using C = GemmCfg<PREC, ROWB, BN>;
  void* bhi = ws_at<void>(ws, g.off_bhi);
  void* blo = ws_at<void>(ws, g.off_blo);
  CUtensorMap mAhi, mAlo, mBhi, mBlo;
  int st = make_map(&mBhi, bhi, g.elem, g.Kpad, g.Opad, C::kBN, ROWB, C::kScaled);
  if (st == B200D2_OK) st = make_map(&mBlo, blo, g.elem, g.Kpad, g.Opad, C::kBN, ROWB, C::kScaled);
  if (GEN) {  // no A planes; the kernel does not read these maps
    mAhi = mBhi;
    mAlo = mBlo;
  } else {
    if (st == B200D2_OK)
      st = make_map(&mAhi, ws_at<void>(ws, g.off_ahi), g.elem, g.Kpad, g.Mpad, C::kBM, ROWB, C::kScaled);
    if (st == B200D2_OK)
      st = make_map(&mAlo, ws_at<void>(ws, g.off_alo), g.elem, g.Kpad, g.Mpad, C::kBM, ROWB, C::kScaled);
  }
  if (st != B200D2_OK) return st;
  const int wl = BN == 256 ? 0 : 1;  // work list of this tile width
  GemmArgs a;
  memset(&a, 0, sizeof(a));
  a.Mrows = g.Mrows;
  a.Mtiles = g.Mpad / C::kBM;
  a.Ntiles = g.Opad / C::kBN;
  a.O = g.O;
  a.T = g.T;
  a.KB = g.Kpad / C::kBK;
  a.accumulate = b.accumulate;
  {
    // Tile order.  m-major re-reads B (all orientations) for every wave of
    // m-tiles: right when B stays in L2.  Otherwise group the m-tiles so a
    // group's A rows (about 48 MB) stay in L2 while B streams once per group.
    const double l2_budget = 48.0 * 1024 * 1024;
    const double b_bytes = (double)g.Opad * g.Kpad * g.elem * C::kPlanes;
    const double a_tile = (double)C::kBM * g.Kpad * g.elem * C::kPlanes;
    a.group_m = 0;
    if (b_bytes > 64.0 * 1024 * 1024 && a.Mtiles > 1)
      a.group_m = std::max(1, std::min(a.Mtiles, (int)(l2_budget / a_tile)));
  }
  const int tiles = U ? U->ntiles[wl] : a.Mtiles * a.Ntiles;
  if (tiles == 0) return B200D2_OK;
  a.split = split > 0 ? std::min(split, g.split_max) : auto_split(tiles, a.KB, g.split_max);
  a.split = std::max(1, std::min(std::min(a.split, a.KB), kMaxSplit));  // the epilogue sums at most kMaxSplit
  a.out = b.d_diff2;
  a.na = ws_at<double>(ws, g.off_na);
  a.na_hl = ws_at<float2>(ws, g.off_nahl);
  a.combine64 = g_combine64.load();
  a.cc = b.score == B200D2_SCORE_CC ? 1 : 0;
  a.keys = ws_at<unsigned long long>(ws, g.off_keys);
  a.status = ws_at<uint32_t>(ws, g.off_status);
  a.inv_sa = ws_at<float>(ws, g.off_sa);
  a.inv_sb = ws_at<float>(ws, g.off_sb);
  a.part = ws_at<float>(ws, g.off_part);
  a.cnt = ws_at<unsigned>(ws, g.off_cnt);
  a.L = Layout{U ? U->parts : nullptr, U ? U->rows : nullptr, U ? U->tiles[wl] : nullptr, U ? U->ntiles[wl] : 0};
  a.wait_ns = g_wait_ns.load() ? g_wait_ns.load() : kWaitLimitNs;
  set_gen_args(a, g, ws);
  constexpr int kSmem = gemm_smem_bytes<C, GEN>();
  // the shared-memory opt-in is a per-device function attribute
  static std::atomic<unsigned long long> attr_dev{0};
  int dev = 0;
  B200D2_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_dev.load() & bit)) {
    B200D2_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<PREC, ROWB, BN, GEN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
    attr_dev.fetch_or(bit);
  }
  const long long items = (long long)tiles * a.split;
  const int grid = (int)std::max(1LL, std::min(items, (long long)num_sms()));
  tc_gemm_kernel<PREC, ROWB, BN, GEN><<<grid, GEN ? kGemmThreadsGen : kGemmThreads, kSmem, s>>>(mAhi, mAlo, mBhi,
                                                                                                  mBlo, a);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

template <int PREC, int ROWB, bool GEN>
static int launch_gemm_pair(const b200d2_batch& b, const TcGeom& g, void* ws, cudaStream_t s,
                            const UnevenTabs* U) {
  using C = GemmCfgPair<PREC, ROWB>;
  CUtensorMap mAhi, mAlo, mBhi, mBlo;
  int st = make_map(&mBhi, ws_at<void>(ws, g.off_bhi), g.elem, g.Kpad, g.Opad, 128, ROWB, C::kScaled);
  if (st == B200D2_OK) st = make_map(&mBlo, ws_at<void>(ws, g.off_blo), g.elem, g.Kpad, g.Opad, 128, ROWB, C::kScaled);
  if (GEN) {  // no A planes; the kernel does not read these maps
    mAhi = mBhi;
    mAlo = mBlo;
  } else {
    if (st == B200D2_OK)
      st = make_map(&mAhi, ws_at<void>(ws, g.off_ahi), g.elem, g.Kpad, g.Mpad, 128, ROWB, C::kScaled);
    if (st == B200D2_OK)
      st = make_map(&mAlo, ws_at<void>(ws, g.off_alo), g.elem, g.Kpad, g.Mpad, 128, ROWB, C::kScaled);
  }
  if (st != B200D2_OK) return st;
  GemmArgs a;
  memset(&a, 0, sizeof(a));
  a.Mrows = g.Mrows;
  a.Mtiles = (g.Mpad + 255) / 256;  // a last half tile reads rows past Mpad as zeros (TMA fill)
  a.Ntiles = g.Opad / 256;
  a.O = g.O;
  a.T = g.T;
  a.KB = g.Kpad / C::kBK;
  a.accumulate = b.accumulate;
  a.split = 1;
  {
    // tile order as for single-CTA tiles, with 256-row m-tiles
    const double b_bytes = (double)g.Opad * g.Kpad * g.elem * C::kPlanes;
    const double a_tile = 256.0 * g.Kpad * g.elem * C::kPlanes;
    a.group_m = 0;
    if (b_bytes > 64.0 * 1024 * 1024 && a.Mtiles > 1)
      a.group_m = std::max(1, std::min(a.Mtiles, (int)(48.0 * 1024 * 1024 / a_tile)));
  }
  a.out = b.d_diff2;
  a.na = ws_at<double>(ws, g.off_na);
  a.na_hl = ws_at<float2>(ws, g.off_nahl);
  a.combine64 = g_combine64.load();
  a.cc = b.score == B200D2_SCORE_CC ? 1 : 0;
  a.keys = ws_at<unsigned long long>(ws, g.off_keys);
  a.status = ws_at<uint32_t>(ws, g.off_status);
  a.inv_sa = ws_at<float>(ws, g.off_sa);
  a.inv_sb = ws_at<float>(ws, g.off_sb);
  a.L = Layout{U ? U->parts : nullptr, U ? U->rows : nullptr, U ? U->tiles[2] : nullptr, U ? U->ntiles[2] : 0};
  a.wait_ns = kWaitLimitNs;  // the pair kernel's waits are not shortened (see b200d2_set_wait_limit_ns)
  set_gen_args(a, g, ws);
  constexpr int kSmem = gemm_smem_bytes<C, GEN>();
  static std::atomic<unsigned long long> attr_dev{0};
  int dev = 0;
  B200D2_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_dev.load() & bit)) {
    B200D2_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_pair_kernel<PREC, ROWB, GEN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
    attr_dev.fetch_or(bit);
  }
  const int tiles = U ? U->ntiles[2] : a.Mtiles * a.Ntiles;
  if (tiles == 0) return B200D2_OK;
  const int pairs = std::max(1, std::min(tiles, num_sms() / 2));
  tc_gemm_pair_kernel<PREC, ROWB, GEN><<<2 * pairs, GEN ? kGemmThreadsGen : kGemmThreads, kSmem, s>>>(
      mAhi, mAlo, mBhi, mBlo, a);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

template <int PREC>
static int launch_gemm(const b200d2_batch& b, const TcGeom& g, void* ws, cudaStream_t s, GemmVariant var,
                       const UnevenTabs* U) {
  if (!U) {  // batch entry points: the process-wide setting fills unset fields
    if (var.row_bytes <= 0) var.row_bytes = g_var_rb.load();
    if (var.bn <= 0) var.bn = g_var_bn.load();
    if (var.split <= 0) var.split = g_var_split.load();
    if (var.pair <= 0) var.pair = g_var_pair.load();
  }
  // CTA pairs by default for uniform batches whose 256 x 256 tiles fill the
  // GPU (one tile per pair of SMs at least); their default rows are 128 bytes
  bool pair = var.pair == 1;
  if (var.pair == 0 && !U && (var.bn <= 0 || var.bn == 256) && var.split <= 1)
    pair = (long long)((g.Mpad + 255) / 256) * (g.Opad / 256) >= num_sms() / 2;
  if (pair && (var.bn <= 0 || var.bn == 256) && var.split <= 1) {
    const int prb = var.row_bytes > 0 ? var.row_bytes : 128;
    if (g.gen)
      return prb == 128 ? launch_gemm_pair<PREC, 128, true>(b, g, ws, s, U)
                        : launch_gemm_pair<PREC, 64, true>(b, g, ws, s, U);
    return prb == 128 ? launch_gemm_pair<PREC, 128, false>(b, g, ws, s, U)
                      : launch_gemm_pair<PREC, 64, false>(b, g, ws, s, U);
  }
  const int rb = var.row_bytes > 0 ? var.row_bytes : gemm_row_bytes();
  // uniform batches too small for CTA pairs: 128-wide tiles while they still
  // fit in one wave (twice the CTAs; at C1 31 instead of 41 us)
  if (var.bn <= 0 && !U && (long long)(g.Mpad / 128) * ((g.Opad + 127) / 128) <= num_sms()) var.bn = 128;
  if (g.gen) {
    if (var.bn == 128)
      return rb == 128 ? launch_gemm_v<PREC, 128, 128, true>(b, g, ws, s, U, var.split)
                       : launch_gemm_v<PREC, 64, 128, true>(b, g, ws, s, U, var.split);
    return rb == 128 ? launch_gemm_v<PREC, 128, 256, true>(b, g, ws, s, U, var.split)
                     : launch_gemm_v<PREC, 64, 256, true>(b, g, ws, s, U, var.split);
  }
  if (var.bn == 128)
    return rb == 128 ? launch_gemm_v<PREC, 128, 128, false>(b, g, ws, s, U, var.split)
                     : launch_gemm_v<PREC, 64, 128, false>(b, g, ws, s, U, var.split);
  return rb == 128 ? launch_gemm_v<PREC, 128, 256, false>(b, g, ws, s, U, var.split)
                   : launch_gemm_v<PREC, 64, 256, false>(b, g, ws, s, U, var.split);
}

template <int PREC>
static int launch_stage(const b200d2_view& v, const b200d2_batch& b, const TcGeom& g, void* ws, int stage,
                        cudaStream_t s, const UnevenTabs* U, GemmVariant var) {
  const PartDev* parts = U ? U->parts : nullptr;
  uint32_t* status = ws_at<uint32_t>(ws, g.off_status);
  int2* xy = ws_at<int2>(ws, g.off_xy);
  int* idx = ws_at<int>(ws, g.off_idx);
  float2* ex = ws_at<float2>(ws, g.off_ex);
  float2* ey = ws_at<float2>(ws, g.off_ey);
  float2* ph = ws_at<float2>(ws, g.off_ph);
  void* bhi = ws_at<void>(ws, g.off_bhi);
  void* blo = ws_at<void>(ws, g.off_blo);
  double* q = ws_at<double>(ws, g.off_q);
  double* wcomp = ws_at<double>(ws, g.off_w);
  double* normx = ws_at<double>(ws, g.off_normx);
  double* na = ws_at<double>(ws, g.off_na);
  float2* na_hl = ws_at<float2>(ws, g.off_nahl);
  void* ahi = ws_at<void>(ws, g.off_ahi);
  void* alo = ws_at<void>(ws, g.off_alo);
  unsigned long long* keys = ws_at<unsigned long long>(ws, g.off_keys);
  constexpr bool kScaled = (PREC == B200D2_PREC_FP16 || PREC == B200D2_PREC_FP16X3);
  float* inv_sa = ws_at<float>(ws, g.off_sa);
  float* inv_sb = ws_at<float>(ws, g.off_sb);
  switch (stage) {
    case 0:
      tc_pixel_list_kernel<<<1, 1024, 0, s>>>(v, g.N_img, xy, idx, status, keys, g.P, b.d_coor_xy,
                                              g.K_c, g.maxR, ws_at<unsigned>(ws, g.off_cnt), g.n_cnt);
      break;
    case 1: {
      const int n = g.T * (g.exw + g.eyw);
      tc_phase_kernel<<<std::max(1, std::min((n + 255) / 256, 1024)), 256, 0, s>>>(
          b.d_trans_x, b.d_trans_y, g.T, g.maxR, ex, ey, U ? U->tab_txy : nullptr);
      count_launch();
      tc_phase2d_kernel<<<dim3((g.Kpad / 2 + 255) / 256, std::min(g.T, 65535)), 256, 0, s>>>(
          ex, ey, xy, g.K_c, g.Kpad / 2, g.T, g.maxR, ph);
      if (g.gen) {
        count_launch();
        tc_phase_compact_kernel<<<1, kCompactThreads, 0, s>>>(
            b.d_trans_x, b.d_trans_y, U ? U->tab_txy : nullptr, g.T, xy, g.K_c, ex, ey, g.maxR,
            ws_at<int2>(ws, g.off_cxy), ws_at<int>(ws, g.off_thdr), ws_at<float2>(ws, g.off_exc),
            ws_at<float2>(ws, g.off_eyc), kGenTabEntries);
      }
      if (kScaled) {  // the particle scales, needed by stage 5 on the same stream
        count_launch();
        tc_scale_a_kernel<<<g.P, 256, 0, s>>>(b.d_real, b.d_imag, b.d_corr, b.img_stride, parts, idx, g.K_c,
                                              inv_sa);
      }
      break;
    }
    case 2: {
      if (kScaled) {
        tc_project_scaled_kernel<PREC><<<g.Opad, 256, 0, s>>>(v, b.d_eulers, g.O, xy, g.K_c, g.Kpad, bhi, blo, q,
                                                              inv_sb);
      } else {
        static_assert(256 % kProjOrients == 0, "orientation groups divide Opad");
        dim3 grid((g.Kpad / 2 + 127) / 128, g.Opad / kProjOrients);
        tc_project_kernel<PREC><<<grid, 128, 0, s>>>(v, b.d_eulers, g.O, xy, g.K_c, g.Kpad, bhi, blo, q,
                                                     g.d_proj_need, g.d_eul_cache);
      }
      break;
    }
    case 3:
      tc_normx_kernel<<<g.P, 256, 0, s>>>(b.d_real, b.d_imag, b.d_corr, b.img_stride, g.N_img, normx, parts,
                                          idx, g.K_c, g.Kq, wcomp, ws_at<float2>(ws, g.off_wx),
                                          kScaled ? inv_sa : nullptr);
      break;
    case 4: {
      // the largest tile (particles x orientations: 64 x 64, 32 x 64, 16 x 64,
      // 16 x 32, 16 x 16) that still gives every SM a CTA
      const int sms = num_sms();
      const int cc = b.score == B200D2_SCORE_CC;
      if (U && U->ntile[0]) {  // uneven batch: only the blocks some particle needs
        const int li = U->nsel >= 0 ? U->nsel : U->nntile[0] >= sms ? 0 : U->nntile[1] >= sms ? 1 : 2;
        if (li == 0)
          B200D2_CUDA_TRY((launch_norma<4, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O, U->ntile[0],
                                              U->nntile[0], U->nperm)));
        else if (li == 1)
          B200D2_CUDA_TRY((launch_norma<2, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O, U->ntile[1],
                                              U->nntile[1], U->nperm)));
        else
          B200D2_CUDA_TRY((launch_norma<1, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O, U->ntile[2],
                                              U->nntile[2], U->nperm)));
        break;
      }
      auto ctas = [&](int cp, int co) { return (long long)((g.O + co - 1) / co) * ((g.P + cp - 1) / cp); };
      if (ctas(64, 64) >= sms)
        B200D2_CUDA_TRY((launch_norma<4, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O)));
      else if (ctas(32, 64) >= sms)
        B200D2_CUDA_TRY((launch_norma<2, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O)));
      else if (ctas(16, 64) >= sms)
        B200D2_CUDA_TRY((launch_norma<1, 4>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O)));
      else if (ctas(16, 32) >= sms)
        B200D2_CUDA_TRY((launch_norma<1, 2>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O)));
      else
        B200D2_CUDA_TRY((launch_norma<1, 1>(s, wcomp, g.Kq, q, g.O, g.P, normx, na, na_hl, cc, g.O)));
      break;
    }
    case 5: {
      if (g.gen) return B200D2_OK;  // A is generated inside the contraction
      // one thread per four complex pixels of a row; warps spread evenly over
      // at most 8-warp blocks; kGenRows rows per block (Mpad is a multiple of 128)
      const int Kh = g.Kpad / 2, warps = (Kh / kGenV + 31) / 32;
      const int nblk = (warps + 7) / 8, bw = (warps + nblk - 1) / nblk;
      const dim3 grid(nblk, g.Mpad / kGenRows);
      const float* isa = kScaled ? inv_sa : nullptr;
      if (U)
        tc_gen_a_kernel<PREC, true><<<grid, 32 * bw, 0, s>>>(b.d_real, b.d_imag, b.d_corr, b.img_stride, idx, g.K_c,
                                                             Kh, ph, g.T, g.Mrows, ahi, alo, parts, U->rows, isa);
      else
        tc_gen_a_kernel<PREC, false><<<grid, 32 * bw, 0, s>>>(b.d_real, b.d_imag, b.d_corr, b.img_stride, idx,
                                                              g.K_c, Kh, ph, g.T, g.Mrows, ahi, alo, parts, nullptr,
                                                              isa);
      break;
    }
    case 6:
      return launch_gemm<PREC>(b, g, ws, s, var, U);
    case 7:
      tc_finalize_kernel<<<(g.P + 127) / 128, 128, 0, s>>>(keys, g.P, b.d_min, b.d_argmin);
      break;
    default:
      return B200D2_ERR_INVALID;
  }
  count_launch();
  return status_from_cuda(cudaGetLastError());
}

const char* tc_stage_name(int precision, int stage);

static int dispatch_stage(const b200d2_view& v, const b200d2_batch& b, int prec, const TcGeom& g, void* ws,
                          int stage, cudaStream_t s, const UnevenTabs* U = nullptr,
                          GemmVariant var = GemmVariant()) {
  const char* name = tc_stage_name(prec, stage);
  NvtxRange range(name ? name : "b200d2 stage");
  switch (prec) {
    case B200D2_PREC_BF16X3: return launch_stage<B200D2_PREC_BF16X3>(v, b, g, ws, stage, s, U, var);
    case B200D2_PREC_TF32X3: return launch_stage<B200D2_PREC_TF32X3>(v, b, g, ws, stage, s, U, var);
    case B200D2_PREC_TF32: return launch_stage<B200D2_PREC_TF32>(v, b, g, ws, stage, s, U, var);
    case B200D2_PREC_FP16X3: return launch_stage<B200D2_PREC_FP16X3>(v, b, g, ws, stage, s, U, var);
    case B200D2_PREC_FP16: return launch_stage<B200D2_PREC_FP16>(v, b, g, ws, stage, s, U, var);
    default: return B200D2_ERR_UNSUPPORTED;
  }
}

static constexpr int kNumStages = 8;

size_t tc_workspace_bytes(const b200d2_view& v, const b200d2_batch& b, int precision, bool allow_split) {
  return make_geom(v, b, precision, -1, allow_split).total;
}

// Where a batch's projections live in its workspace and what they were
// computed from, for the single-particle entry point's projection cache:
// false for the FP16 forms (their projection stage also rescales per call)
// and for projections of fewer than 2^20 samples, which take less time than
// the check that would skip them.
bool tc_projection_layout(const b200d2_view& v, const b200d2_batch& b, int precision, std::vector<uint64_t>& key) {
  if (precision == B200D2_PREC_FP16 || precision == B200D2_PREC_FP16X3) return false;
  const TcGeom g = make_geom(v, b, precision);
  if ((long long)g.O * g.K_c < (1LL << 20)) return false;
  key.insert(key.end(), {(uint64_t)precision, (uint64_t)g.elem, (uint64_t)g.terms, (uint64_t)g.K_c,
                         (uint64_t)g.Kpad, (uint64_t)g.Kq, (uint64_t)g.O, (uint64_t)g.Opad, (uint64_t)g.maxR,
                         (uint64_t)g.off_xy, (uint64_t)g.off_bhi, (uint64_t)g.off_blo, (uint64_t)g.off_q,
                         (uint64_t)g.total});
  return true;
}

const char* tc_stage_name(int precision, int stage) {
  static const char* bf16[] = {"tc_pixel_list_kernel", "tc_phase_kernel", "tc_project_kernel<bf16x3>",
                               "tc_normx_kernel", "tc_norma_kernel", "tc_gen_a_kernel<bf16x3>",
                               "tc_gemm[_pair]_kernel<bf16x3>", "tc_finalize_kernel"};
  static const char* tf3[] = {"tc_pixel_list_kernel", "tc_phase_kernel", "tc_project_kernel<tf32x3>",
                              "tc_normx_kernel", "tc_norma_kernel", "tc_gen_a_kernel<tf32x3>",
                              "tc_gemm[_pair]_kernel<tf32x3>", "tc_finalize_kernel"};
  static const char* tf1[] = {"tc_pixel_list_kernel", "tc_phase_kernel", "tc_project_kernel<tf32>",
                              "tc_normx_kernel", "tc_norma_kernel", "tc_gen_a_kernel<tf32>",
                              "tc_gemm[_pair]_kernel<tf32>", "tc_finalize_kernel"};
  // stage 1 also launches tc_phase2d_kernel, tc_phase_compact_kernel (when
  // the contraction generates A) and, in the FP16 forms, tc_scale_a_kernel;
  // in the FP16 forms stage 2 is the two-pass tc_project_scaled_kernel
  static const char* h3[] = {"tc_pixel_list_kernel", "tc_phase_kernel", "tc_project_scaled_kernel<fp16x3>",
                             "tc_normx_kernel", "tc_norma_kernel", "tc_gen_a_kernel<fp16x3>",
                             "tc_gemm[_pair]_kernel<fp16x3>", "tc_finalize_kernel"};
  static const char* h1[] = {"tc_pixel_list_kernel", "tc_phase_kernel", "tc_project_scaled_kernel<fp16>",
                             "tc_normx_kernel", "tc_norma_kernel", "tc_gen_a_kernel<fp16>",
                             "tc_gemm[_pair]_kernel<fp16>", "tc_finalize_kernel"};
  if (stage < 0 || stage >= kNumStages) return nullptr;
  // with the operand generated inside the contraction, stage 5 launches nothing
  if (stage == 5 && is_tc_precision(precision) && g_operand_gen.load()) return "(A operand: generated in the contraction)";
  if (precision == B200D2_PREC_BF16X3) return bf16[stage];
  if (precision == B200D2_PREC_TF32X3) return tf3[stage];
  if (precision == B200D2_PREC_TF32) return tf1[stage];
  if (precision == B200D2_PREC_FP16X3) return h3[stage];
  if (precision == B200D2_PREC_FP16) return h1[stage];
  return nullptr;
}

static int check_tc(const b200d2_view& v, const b200d2_batch& b) {
  if ((long long)b.O * b.T >= 0xffffffffLL) return B200D2_ERR_UNSUPPORTED;  // argmin index is 32-bit
  if (v.maxR > 4096) return B200D2_ERR_UNSUPPORTED;
  return B200D2_OK;
}

int tc_run_stage(const b200d2_view& v, const b200d2_batch& b, int precision, int stage, void* ws,
                 size_t ws_bytes, cudaStream_t s, bool allow_split) {
  int st = check_tc(v, b);
  if (st != B200D2_OK) return st;
  const TcGeom g = make_geom(v, b, precision, -1, allow_split);
  if (ws_bytes < g.total) return B200D2_ERR_INVALID;
  return dispatch_stage(v, b, precision, g, ws, stage, s);
}

// Side stream (and fork/join events) paired with a caller stream on the
// current device.  Calls on one caller stream are ordered by that stream, so
// reusing the pair's events across calls is safe; fork/join through events is
// also what stream capture records into a graph.
struct SidePair {
  int device;
  cudaStream_t user, side;
  cudaEvent_t fork, mid, join;
};

static std::mutex g_side_mu;
static std::vector<SidePair> g_side;

static int side_for(cudaStream_t user, SidePair* out) {
  int dev = 0;
  B200D2_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_side_mu);
  for (const SidePair& sp : g_side)
    if (sp.device == dev && sp.user == user) {
      *out = sp;
      return B200D2_OK;
    }
  SidePair sp;
  sp.device = dev;
  sp.user = user;
  B200D2_CUDA_TRY(cudaStreamCreateWithFlags(&sp.side, cudaStreamNonBlocking));
  B200D2_CUDA_TRY(cudaEventCreateWithFlags(&sp.fork, cudaEventDisableTiming));
  B200D2_CUDA_TRY(cudaEventCreateWithFlags(&sp.mid, cudaEventDisableTiming));
  B200D2_CUDA_TRY(cudaEventCreateWithFlags(&sp.join, cudaEventDisableTiming));
  g_side.push_back(sp);
  *out = sp;
  return B200D2_OK;
}

// The whole pipeline of one batch on stream s (forking to the side stream
// paired with s and joining back).
static int tc_launch_pipeline(const b200d2_view& v, const b200d2_batch& b, int precision, const TcGeom& g, void* ws,
                              cudaStream_t s) {
  int st = B200D2_OK;
  SidePair sp;
  st = side_for(s, &sp);
  if (st != B200D2_OK) return st;
  // caller stream: pixel list -> projections -> (normX) -> normA; side
  // stream: phase tables -> normX -> operand generation; normA waits for
  // normX, the contraction for both streams.
  st = dispatch_stage(v, b, precision, g, ws, 0, s);
  if (st != B200D2_OK) return st;
  B200D2_CUDA_TRY(cudaEventRecord(sp.fork, s));
  B200D2_CUDA_TRY(cudaStreamWaitEvent(sp.side, sp.fork, 0));
  st = dispatch_stage(v, b, precision, g, ws, 1, sp.side);
  if (st == B200D2_OK) st = dispatch_stage(v, b, precision, g, ws, 3, sp.side);
  const cudaError_t rm = cudaEventRecord(sp.mid, sp.side);
  if (st == B200D2_OK) st = dispatch_stage(v, b, precision, g, ws, 5, sp.side);
  const cudaError_t rj = cudaEventRecord(sp.join, sp.side);
  if (st != B200D2_OK) return st;
  if (rm != cudaSuccess) return status_from_cuda(rm);
  if (rj != cudaSuccess) return status_from_cuda(rj);
  st = dispatch_stage(v, b, precision, g, ws, 2, s);
  if (st != B200D2_OK) return st;
  B200D2_CUDA_TRY(cudaStreamWaitEvent(s, sp.mid, 0));
  st = dispatch_stage(v, b, precision, g, ws, 4, s);
  if (st != B200D2_OK) return st;
  B200D2_CUDA_TRY(cudaStreamWaitEvent(s, sp.join, 0));
  st = dispatch_stage(v, b, precision, g, ws, 6, s);
  if (st == B200D2_OK) st = dispatch_stage(v, b, precision, g, ws, 7, s);
  return st;
}

// Cached CUDA graphs of the batch pipeline.  A call's launches are fixed by
// its arguments (view, batch fields and pointers, precision, workspace) and
// the process-wide settings (contraction variant, combine, operand mode,
// wait limit) on a given device and stream: the second call with the same
// signature captures the pipeline once into a graph, later ones launch that
// graph (one host call instead of about a dozen launches, event records and
// waits).  Calls whose stream is being captured by the caller run the
// launches directly, so that they become part of the caller's graph.
static std::atomic<int> g_batch_graphs{1};  // b200d2_set_batch_graphs

struct BatchGraph {
  std::vector<uint64_t> key;
  int seen = 0;
  unsigned long long last = 0;
  unsigned launches = 0;  // kernels in the graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
static std::mutex g_graph_mu;
static std::vector<BatchGraph> g_graphs;
static unsigned long long g_graph_clock = 0;
constexpr size_t kMaxBatchGraphs = 32;

static std::vector<uint64_t> batch_key(const b200d2_view& v, const b200d2_batch& b, int precision, const void* ws,
                                       size_t ws_bytes, cudaStream_t s, int dev) {
  auto u = [](const void* p) { return (uint64_t)(uintptr_t)p; };
  auto f = [](float x) {
    uint32_t r;
    memcpy(&r, &x, 4);
    return (uint64_t)r;
  };
  return {(uint64_t)dev, u(s), u(ws), (uint64_t)ws_bytes, (uint64_t)precision,
          // view
          (uint64_t)v.mdlX, (uint64_t)v.mdlXY, (uint64_t)v.mdlZ, (uint64_t)v.imgX, (uint64_t)v.imgY,
          (uint64_t)v.imgZ, (uint64_t)(uint32_t)v.mdlInitY, (uint64_t)(uint32_t)v.mdlInitZ, (uint64_t)v.maxR,
          (uint64_t)v.maxR2, (uint64_t)v.maxR2_padded, f(v.padding_factor), v.tex_re, v.tex_im, u(v.lin_re),
          u(v.lin_im), (uint64_t)v.interp, v.tex_c,
          // batch
          u(b.d_eulers), (uint64_t)b.O, u(b.d_trans_x), u(b.d_trans_y), (uint64_t)b.T, (uint64_t)b.P,
          (uint64_t)b.N_img, u(b.d_real), u(b.d_imag), u(b.d_corr), (uint64_t)b.img_stride, u(b.d_diff2),
          (uint64_t)b.accumulate, u(b.d_min), u(b.d_argmin), u(b.d_coor_xy), (uint64_t)b.n_listed,
          (uint64_t)b.score,
          // process-wide settings read by the launches
          (uint64_t)g_var_rb.load(), (uint64_t)g_var_bn.load(), (uint64_t)g_var_split.load(),
          (uint64_t)g_var_pair.load(), (uint64_t)g_combine64.load(), (uint64_t)g_operand_gen.load(),
          (uint64_t)g_wait_ns.load()};
}

// A private capture stream per device.
static cudaStream_t capture_stream(int dev) {
  static std::mutex mu;
  static std::map<int, cudaStream_t> streams;
  std::lock_guard<std::mutex> lk(mu);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  streams[dev] = cs;
  return cs;
}

unsigned long long launch_counter();
void uncount_launch(unsigned n);

int tc_run(const b200d2_view& v, const b200d2_batch& b, int precision, void* ws, size_t ws_bytes,
           cudaStream_t s, const int* d_proj_need, float* d_eul_cache) {
  NvtxRange range("b200d2_diff2_coarse_batch");
  int st = check_tc(v, b);
  if (st != B200D2_OK) return st;
  TcGeom g = make_geom(v, b, precision);
  g.d_proj_need = d_proj_need;
  g.d_eul_cache = d_eul_cache;
  if (ws_bytes < g.total) return B200D2_ERR_INVALID;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!g_batch_graphs.load() || cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return tc_launch_pipeline(v, b, precision, g, ws, s);
  int dev = 0;
  B200D2_CUDA_TRY(cudaGetDevice(&dev));
  std::vector<uint64_t> key = batch_key(v, b, precision, ws, ws_bytes, s, dev);
  key.push_back((uint64_t)(uintptr_t)d_proj_need);
  key.push_back((uint64_t)(uintptr_t)d_eul_cache);
  std::unique_lock<std::mutex> lk(g_graph_mu);
  BatchGraph* e = nullptr;
  for (BatchGraph& x : g_graphs)
    if (x.key == key) {
      e = &x;
      break;
    }
  if (!e) {
    if (g_graphs.size() >= kMaxBatchGraphs) {  // evict the least recently used signature
      size_t lru = 0;
      for (size_t i = 1; i < g_graphs.size(); ++i)
        if (g_graphs[i].last < g_graphs[lru].last) lru = i;
      if (g_graphs[lru].exec) cudaGraphExecDestroy(g_graphs[lru].exec);
      if (g_graphs[lru].graph) cudaGraphDestroy(g_graphs[lru].graph);
      g_graphs.erase(g_graphs.begin() + (long)lru);
    }
    g_graphs.push_back(BatchGraph());
    e = &g_graphs.back();
    e->key = key;
  }
  e->last = ++g_graph_clock;
  if (!e->exec && e->seen == 0) {  // first call with this signature: launch directly
    e->seen = 1;
    lk.unlock();
    return tc_launch_pipeline(v, b, precision, g, ws, s);
  }
  if (!e->exec) {  // second call: capture once
    cudaStream_t cs = capture_stream(dev);
    if (!cs) {
      lk.unlock();
      return tc_launch_pipeline(v, b, precision, g, ws, s);
    }
    const unsigned long long l0 = launch_counter();
    st = status_from_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    if (st == B200D2_OK) {
      const int st2 = tc_launch_pipeline(v, b, precision, g, ws, cs);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
      st = st2 != B200D2_OK ? st2 : status_from_cuda(ce);
      if (st == B200D2_OK) st = status_from_cuda(cudaGraphInstantiate(&e->exec, graph, 0));
      if (st == B200D2_OK) {
        e->graph = graph;
      } else if (graph) {
        cudaGraphDestroy(graph);
      }
    }
    // the launches were counted while capturing; the graph launch below counts them
    e->launches = (unsigned)(launch_counter() - l0);
    uncount_launch(e->launches);
    if (st != B200D2_OK || !e->exec) {  // capture not possible: stay with direct launches
      e->exec = nullptr;
      e->seen = 1;
      lk.unlock();
      return tc_launch_pipeline(v, b, precision, g, ws, s);
    }
  }
  const cudaError_t le = cudaGraphLaunch(e->exec, s);
  const unsigned n = e->launches;
  lk.unlock();
  if (le != cudaSuccess) return status_from_cuda(le);
  count_launch(n);
  return B200D2_OK;
}

// ------------------------------------------------------------------ plans
// Autotuner cache: contraction variant chosen for a problem signature.
struct TuneKey {
  int prec, Kpad, O, mtiles, ntiles;
  bool operator<(const TuneKey& o) const {
    return std::tie(prec, Kpad, O, mtiles, ntiles) < std::tie(o.prec, o.Kpad, o.O, o.mtiles, o.ntiles);
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, GemmVariant> g_tune_cache;

}  // namespace b200d2

struct b200d2_plan {
  b200d2_view view;
  b200d2_batch batch;  // shared geometry (T = number of phase tables), min/argmin outputs
  int prec = 0, flags = 0;
  b200d2::GemmVariant var;  // contraction variant in use
  b200d2::TcGeom g;
  b200d2::UnevenTabs U;
  void* ws = nullptr;
  b200d2::PartDev* d_parts = nullptr;
  int4* d_rows = nullptr;
  int2* d_tiles = nullptr;     // work list, 256-wide tiles
  int2* d_tiles128 = nullptr;  // work list, 128-wide tiles
  int2* d_tiles_pair = nullptr;  // work list, 256 x 256 tiles of CTA pairs
  int2* d_ntile[3] = {nullptr, nullptr, nullptr};  // norm kernel work lists
  int* d_nperm = nullptr;                         // particle order of their tiles
  float2* d_txy = nullptr;
  int* d_inv = nullptr;
  float* d_eul_perm = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  b200d2_plan_info info;
};

namespace b200d2 {

static void plan_free(b200d2_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->stream) cudaStreamDestroy(p->stream);
  for (void* d : {(void*)p->ws, (void*)p->d_parts, (void*)p->d_rows, (void*)p->d_tiles, (void*)p->d_tiles128,
                  (void*)p->d_tiles_pair, (void*)p->d_ntile[0], (void*)p->d_ntile[1], (void*)p->d_ntile[2],
                  (void*)p->d_nperm, (void*)p->d_txy, (void*)p->d_inv, (void*)p->d_eul_perm})
    if (d) cudaFree(d);
  delete p;
}

// All stages in order on one stream (the form that is captured).
static int plan_pipeline(b200d2_plan* p, cudaStream_t s, GemmVariant var) {
  int st = B200D2_OK;
  for (int i = 0; i < kNumStages && st == B200D2_OK; ++i)
    st = dispatch_stage(p->view, p->batch, p->prec, p->g, p->ws, i, s, &p->U, var);
  return st;
}

// Best of `reps` timed launches of one stage of the plan (its own stream).
static double time_stage(b200d2_plan* p, int stage, int reps) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 1e30;
  for (int r = 0; r < reps + 1; ++r) {  // the first launch is not counted
    cudaEventRecord(a, p->stream);
    const int st = dispatch_stage(p->view, p->batch, p->prec, p->g, p->ws, stage, p->stream, &p->U, p->var);
    cudaEventRecord(b, p->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (st == B200D2_OK && r > 0) best = std::min(best, (double)ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

static double time_gemm(b200d2_plan* p, GemmVariant var, int reps) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 1e30;
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(a, p->stream);
    int st = dispatch_stage(p->view, p->batch, p->prec, p->g, p->ws, 6, p->stream, &p->U, var);
    cudaEventRecord(b, p->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (st == B200D2_OK) best = std::min(best, (double)ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace b200d2

extern "C" int b200d2_plan_create(const b200d2_view* view, const float* d_eulers, int O_all, int N_img,
                                  const b200d2_particle_desc* parts, int P, int precision, int flags,
                                  double* d_min, long long* d_argmin, b200d2_plan** out) {
  using namespace b200d2;
  if (!view || !d_eulers || !parts || !out || P <= 0 || O_all <= 0 || N_img <= 0) return B200D2_ERR_INVALID;
  *out = nullptr;
  if (!is_tc_precision(precision)) return B200D2_ERR_UNSUPPORTED;
  if (view->mdlZ == 0 || (long long)view->imgX * view->imgY < N_img) return B200D2_ERR_INVALID;
  for (int i = 0; i < P; ++i) {
    const b200d2_particle_desc& d = parts[i];
    if (!d.d_real || !d.d_imag || !d.d_corr || !d.d_diff2 || !d.h_trans_x || !d.h_trans_y) return B200D2_ERR_INVALID;
    if (d.O <= 0 || d.T <= 0 || d.O > O_all) return B200D2_ERR_INVALID;
    if ((long long)d.O * d.T >= 0xffffffffLL) return B200D2_ERR_UNSUPPORTED;
    if (d.h_orient)
      for (int k = 0; k < d.O; ++k)
        if (d.h_orient[k] < 0 || d.h_orient[k] >= O_all) return B200D2_ERR_INVALID;
  }
  b200d2_plan* p = new b200d2_plan();
  p->view = *view;
  p->prec = precision;
  p->flags = flags;

  // column position of every orientation: identity, or sorted by the
  // position of the viewing direction (third column of the Euler matrix,
  // which is the same for all in-plane angles of one direction) along a
  // Hilbert curve over (z, azimuth) quantised to 16 bits each (on C4, 3 %
  // fewer CTA-pair tiles than the Morton order of the same coordinates)
  std::vector<int> pos(O_all), perm(O_all);
  for (int o = 0; o < O_all; ++o) perm[o] = o;
  std::vector<float> h_eul;
  if (flags & B200D2_PLAN_REORDER) {
    h_eul.resize((size_t)O_all * 9);
    if (cudaMemcpy(h_eul.data(), d_eulers, h_eul.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
      delete p;
      return B200D2_ERR_CUDA;
    }
    std::vector<uint64_t> key(O_all);
    for (int o = 0; o < O_all; ++o) {
      const float* e = &h_eul[(size_t)o * 9];
      const double dz = std::max(-1.0, std::min(1.0, (double)e[8]));
      const double ph = atan2((double)e[5], (double)e[2]);  // in (-pi, pi]
      const uint32_t u = (uint32_t)std::min(65535.0, (dz + 1.0) * 0.5 * 65536.0);
      const uint32_t w = (uint32_t)std::min(65535.0, (ph / (2 * 3.14159265358979323846) + 0.5) * 65536.0);
      // Hilbert index of (u, w) on a 65536 x 65536 grid
      uint32_t x = u, y = w;
      uint64_t d = 0;
      for (uint32_t sq = 1u << 15; sq > 0; sq >>= 1) {
        const uint32_t rx = (x & sq) ? 1u : 0u, ry = (y & sq) ? 1u : 0u;
        d += (uint64_t)sq * sq * ((3u * rx) ^ ry);
        if (ry == 0) {  // rotate the quadrant
          if (rx == 1) {
            x = sq - 1 - (x & (sq - 1)) + (x & ~(2 * sq - 1));
            y = sq - 1 - (y & (sq - 1)) + (y & ~(2 * sq - 1));
          }
          const uint32_t t = x;
          x = y;
          y = t;
        }
      }
      key[o] = d;
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int c) { return key[a] < key[c]; });
  }
  for (int c = 0; c < O_all; ++c) pos[perm[c]] = c;
  // particle order: by the median column of their subsets
  std::vector<int> ord(P);
  for (int i = 0; i < P; ++i) ord[i] = i;
  if (flags & B200D2_PLAN_REORDER) {
    std::vector<double> mid(P);
    for (int i = 0; i < P; ++i) {
      const b200d2_particle_desc& d = parts[i];
      std::vector<int> c(d.O);
      for (int k = 0; k < d.O; ++k) c[k] = pos[d.h_orient ? d.h_orient[k] : k];
      std::nth_element(c.begin(), c.begin() + d.O / 2, c.end());
      mid[i] = c[d.O / 2];
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return mid[a] < mid[c]; });
    // then a nearest-neighbour chain over the particles' sets of 128-column
    // blocks (Hamming distance, ties by distance in the median order), so that
    // particles sharing an m-tile need similar column blocks: on C4 (1024
    // particles) 5427 instead of 6034 CTA-pair tiles.  Quadratic in P, so
    // larger plans keep the median order.
    constexpr int kChainMaxParticles = 4096;
    if (P > 2 && P <= kChainMaxParticles) {
      const int nb = (O_all + 127) / 128, W = (nb + 63) / 64;
      std::vector<uint64_t> bits((size_t)P * W, 0ull);
      for (int i = 0; i < P; ++i) {
        const b200d2_particle_desc& d = parts[i];
        for (int k = 0; k < d.O; ++k) {
          const int blk = pos[d.h_orient ? d.h_orient[k] : k] / 128;
          bits[(size_t)i * W + blk / 64] |= 1ull << (blk % 64);
        }
      }
      std::vector<int> rank(P);
      for (int r = 0; r < P; ++r) rank[ord[r]] = r;
      std::vector<char> used(P, 0);
      std::vector<int> chain;
      chain.reserve(P);
      int cur = ord[0];
      used[cur] = 1;
      chain.push_back(cur);
      for (int step = 1; step < P; ++step) {
        int best = -1;
        long long best_key = 0;
        for (int j = 0; j < P; ++j) {
          if (used[j]) continue;
          int dist = 0;
          for (int w = 0; w < W; ++w) dist += __builtin_popcountll(bits[(size_t)cur * W + w] ^ bits[(size_t)j * W + w]);
          const long long k = ((long long)dist << 32) + std::abs(rank[j] - rank[cur]);
          if (best < 0 || k < best_key) {
            best = j;
            best_key = k;
          }
        }
        used[best] = 1;
        chain.push_back(best);
        cur = best;
      }
      ord.swap(chain);
    }
  }

  // distinct translation sets -> phase tables; rows (particle, t, table)
  std::map<std::vector<std::pair<uint32_t, uint32_t>>, int> sets;
  std::vector<float2> txy;
  std::vector<int> tab0(P);
  std::vector<int4> rows;
  std::vector<PartDev> hp(P);
  long long evals = 0;
  for (int oi = 0; oi < P; ++oi) {
    const int i = ord[oi];
    const b200d2_particle_desc& d = parts[i];
    std::vector<std::pair<uint32_t, uint32_t>> key(d.T);
    for (int t = 0; t < d.T; ++t) {
      uint32_t a, c;
      memcpy(&a, &d.h_trans_x[t], 4);
      memcpy(&c, &d.h_trans_y[t], 4);
      key[t] = {a, c};
    }
    auto it = sets.find(key);
    if (it == sets.end()) {
      it = sets.emplace(key, (int)txy.size()).first;
      for (int t = 0; t < d.T; ++t) txy.push_back(make_float2(d.h_trans_x[t], d.h_trans_y[t]));
    }
    tab0[i] = it->second;
    hp[i].re = d.d_real;
    hp[i].im = d.d_imag;
    hp[i].corr = d.d_corr;
    hp[i].out = d.d_diff2;
    hp[i].T = d.T;
    hp[i].O = d.O;
    hp[i].row0 = (int)rows.size();
    hp[i].pad = 0;
    for (int t = 0; t < d.T; ++t) rows.push_back(make_int4(i, t, tab0[i] + t, 0));
    evals += (long long)d.O * d.T;
  }
  const int Mrows = (int)rows.size();
  const int Mtiles = (Mrows + 127) / 128, Ntiles = (O_all + 255) / 256, Ntiles128 = (O_all + 127) / 128;

  // orientation -> local index maps, and the n-tiles each particle needs
  std::vector<int> inv((size_t)P * O_all, -1);
  std::vector<std::vector<char>> need_n(P, std::vector<char>(Ntiles128, 0));  // 128-wide column blocks
  for (int i = 0; i < P; ++i) {
    const b200d2_particle_desc& d = parts[i];
    for (int k = 0; k < d.O; ++k) {
      const int c = pos[d.h_orient ? d.h_orient[k] : k];
      inv[(size_t)i * O_all + c] = k;
      need_n[i][c / 128] = 1;
    }
  }
  // work lists: (m tile, n tile) pairs some particle of the m tile needs,
  // m-major, for 256- and 128-wide tiles
  std::vector<int2> tiles, tiles128, tiles_pair;
  for (int mt = 0; mt < (Mtiles + 1) / 2; ++mt) {  // 256-row m-tiles for CTA pairs
    const int r0 = mt * 256, r1 = std::min(Mrows, r0 + 256);
    std::vector<char> un(Ntiles128, 0);
    for (int r = r0; r < r1; ++r)
      if (r == r0 || rows[r].x != rows[r - 1].x)
        for (int n = 0; n < Ntiles128; ++n) un[n] |= need_n[rows[r].x][n];
    for (int n = 0; n < Ntiles; ++n)
      if (un[2 * n] || (2 * n + 1 < Ntiles128 && un[2 * n + 1])) tiles_pair.push_back(make_int2(mt, n));
  }
  for (int mt = 0; mt < Mtiles; ++mt) {
    const int r0 = mt * 128, r1 = std::min(Mrows, r0 + 128);
    std::vector<char> un(Ntiles128, 0);
    for (int r = r0; r < r1; ++r)
      if (r == r0 || rows[r].x != rows[r - 1].x)
        for (int n = 0; n < Ntiles128; ++n) un[n] |= need_n[rows[r].x][n];
    for (int n = 0; n < Ntiles; ++n)
      if (un[2 * n] || (2 * n + 1 < Ntiles128 && un[2 * n + 1])) tiles.push_back(make_int2(mt, n));
    for (int n = 0; n < Ntiles128; ++n)
      if (un[n]) tiles128.push_back(make_int2(mt, n));
  }

  b200d2_batch& b = p->batch;
  memset(&b, 0, sizeof(b));
  b.d_eulers = d_eulers;
  if (flags & B200D2_PLAN_REORDER) {  // orientations in column order
    std::vector<float> pe((size_t)O_all * 9);
    for (int c = 0; c < O_all; ++c) memcpy(&pe[(size_t)c * 9], &h_eul[(size_t)perm[c] * 9], 9 * sizeof(float));
    if (cudaMalloc(&p->d_eul_perm, pe.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(p->d_eul_perm, pe.data(), pe.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      plan_free(p);
      return B200D2_ERR_OOM;
    }
    b.d_eulers = p->d_eul_perm;
  }
  b.O = O_all;
  b.T = (int)txy.size();  // number of phase tables
  b.P = P;
  b.N_img = N_img;
  b.d_real = parts[0].d_real;  // unused by the tabled kernels; kept valid
  b.d_imag = parts[0].d_imag;
  b.d_corr = parts[0].d_corr;
  b.img_stride = N_img;
  b.d_diff2 = parts[0].d_diff2;
  b.accumulate = (flags & B200D2_PLAN_ACCUMULATE) ? 1 : 0;
  b.d_min = d_min;
  b.d_argmin = d_argmin;
  p->g = make_geom(*view, b, precision, Mrows);

  int st = B200D2_OK;
  auto upload = [&](void** dst, const void* src, size_t bytes) {
    if (st != B200D2_OK) return;
    cudaError_t e = cudaMalloc(dst, std::max(bytes, (size_t)16));
    if (e == cudaSuccess && bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    st = status_from_cuda(e);
  };
  st = status_from_cuda(cudaMalloc(&p->ws, p->g.total));
  upload(reinterpret_cast<void**>(&p->d_rows), rows.data(), rows.size() * sizeof(int4));
  upload(reinterpret_cast<void**>(&p->d_tiles), tiles.data(), tiles.size() * sizeof(int2));
  upload(reinterpret_cast<void**>(&p->d_tiles128), tiles128.data(), tiles128.size() * sizeof(int2));
  upload(reinterpret_cast<void**>(&p->d_tiles_pair), tiles_pair.data(), tiles_pair.size() * sizeof(int2));
  // the norm kernel's work lists, particle tiles in plan order (particles
  // chained by the column blocks they need share tiles)
  std::vector<int2> nlist[3];
  norma_lists(P, O_all, [&](int pl, int blk) { return need_n[ord[pl]][blk]; }, nlist);
  for (int li = 0; li < 3; ++li)
    upload(reinterpret_cast<void**>(&p->d_ntile[li]), nlist[li].data(), nlist[li].size() * sizeof(int2));
  upload(reinterpret_cast<void**>(&p->d_nperm), ord.data(), ord.size() * sizeof(int));
  upload(reinterpret_cast<void**>(&p->d_txy), txy.data(), txy.size() * sizeof(float2));
  upload(reinterpret_cast<void**>(&p->d_inv), inv.data(), inv.size() * sizeof(int));
  if (st == B200D2_OK)
    for (int i = 0; i < P; ++i) hp[i].inv = p->d_inv + (size_t)i * O_all;
  upload(reinterpret_cast<void**>(&p->d_parts), hp.data(), hp.size() * sizeof(PartDev));
  if (st == B200D2_OK) st = status_from_cuda(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  if (st != B200D2_OK) {
    plan_free(p);
    return st;
  }
  p->U = UnevenTabs{p->d_parts,
                    p->d_rows,
                    {p->d_tiles, p->d_tiles128, p->d_tiles_pair},
                    {(int)tiles.size(), (int)tiles128.size(), (int)tiles_pair.size()},
                    p->d_txy,
                    (int)txy.size(),
                    Mrows,
                    {p->d_ntile[0], p->d_ntile[1], p->d_ntile[2]},
                    {(int)nlist[0].size(), (int)nlist[1].size(), (int)nlist[2].size()},
                    p->d_nperm,
                    -1};

  memset(&p->info, 0, sizeof(p->info));
  p->info.P = P;
  p->info.O_all = O_all;
  p->info.rows = Mrows;
  p->info.tiles = (int)tiles.size();
  p->info.tiles_dense = Mtiles * Ntiles;
  p->info.evals = evals;
  p->info.stages = kNumStages;
  p->info.tiles_n128 = (int)tiles128.size();
  p->info.tiles_pair = (int)tiles_pair.size();
  for (int li = 0; li < 3; ++li) p->info.norm_tiles[li] = (int)nlist[li].size();
  p->info.workspace_bytes = p->g.total + rows.size() * sizeof(int4) +
                            (tiles.size() + tiles128.size() + tiles_pair.size()) * sizeof(int2) +
                            txy.size() * sizeof(float2) + inv.size() * sizeof(int) + hp.size() * sizeof(PartDev) +
                            (nlist[0].size() + nlist[1].size() + nlist[2].size()) * sizeof(int2) +
                            ord.size() * sizeof(int);

  // warm run (also sets kernel attributes outside any capture)
  // without the autotuner a plan takes the process-wide variant
  // (b200d2_set_gemm_variant), single-CTA 256-wide tiles by default
  p->var = GemmVariant();
  p->var.row_bytes = g_var_rb.load() > 0 ? g_var_rb.load() : gemm_row_bytes();
  p->var.bn = g_var_bn.load() > 0 ? g_var_bn.load() : 256;
  p->var.split = g_var_split.load() > 0 ? std::min(g_var_split.load(), p->g.split_max) : 1;
  p->var.pair = g_var_pair.load() == 1 && p->var.bn == 256 && p->var.split == 1 ? 1 : 2;
  st = plan_pipeline(p, p->stream, p->var);
  if (st == B200D2_OK) st = status_from_cuda(cudaStreamSynchronize(p->stream));
  if (st == B200D2_OK && (flags & B200D2_PLAN_AUTOTUNE)) {
    // autotuner: time every (k-block row width, tile width, k-split) variant
    // on this plan's own work lists and keep the fastest; results are cached
    // per problem signature for later plans
    const TuneKey key{precision, p->g.Kpad, O_all, Mtiles, (int)tiles.size()};
    bool cached = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        p->var = it->second;
        cached = true;
      }
    }
    if (!cached) {
      std::vector<GemmVariant> cand;
      const int sms = num_sms();
      for (int rb : {64, 128}) {  // CTA-pair 256 x 256 tiles
        GemmVariant v;
        v.row_bytes = rb;
        v.bn = 256;
        v.split = 1;
        v.pair = 1;
        cand.push_back(v);
      }
      for (int rb : {64, 128})
        for (int bn : {256, 128}) {
          const int nt = bn == 256 ? (int)tiles.size() : (int)tiles128.size();
          for (int sp = 1; sp <= p->g.split_max; sp *= 2) {
            if (sp > 1 && (long long)nt * sp > 2LL * sms) break;  // splits only while the GPU is not full
            GemmVariant v;
            v.row_bytes = rb;
            v.bn = bn;
            v.split = sp;
            v.pair = 2;
            cand.push_back(v);
          }
        }
      double best = 1e30;
      int n = 0;
      for (const GemmVariant& v : cand) {
        time_gemm(p, v, 1);  // first launch of a variant sets its attributes
        const double ms = time_gemm(p, v, 3);
        if (n < B200D2_PLAN_MAX_VARIANTS) {
          p->info.tuned_variant[n][0] = v.row_bytes;
          p->info.tuned_variant[n][1] = v.bn;
          p->info.tuned_variant[n][2] = v.split;
          p->info.tuned_variant[n][3] = v.pair;
          p->info.tuned_ms[n] = ms;
          ++n;
        }
        if (ms < best) {
          best = ms;
          p->var = v;
        }
      }
      p->info.n_tuned = n;
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune_cache[key] = p->var;
    }
    // the norm stage's particle-tile height: smaller tiles skip more blocks
    // that no particle of the tile needs, larger ones reuse more operands
    if (st == B200D2_OK) {
      double best = 1e30;
      int best_li = -1;
      for (int li = 0; li < 3 && st == B200D2_OK; ++li) {
        p->U.nsel = li;
        const double ms = time_stage(p, 4, 3);
        p->info.norm_tuned_ms[li] = ms;
        if (ms < best) {
          best = ms;
          best_li = li;
        }
      }
      p->U.nsel = best_li;
    }
    // leave the outputs as one full run with the chosen variant produces them
    st = plan_pipeline(p, p->stream, p->var);
    if (st == B200D2_OK) st = status_from_cuda(cudaStreamSynchronize(p->stream));
  }
  {
    const int li = p->U.nsel >= 0 ? p->U.nsel
                   : p->U.nntile[0] >= num_sms() ? 0 : p->U.nntile[1] >= num_sms() ? 1 : 2;
    p->info.norm_tile_p = 64 >> li;
  }
  p->info.row_bytes = p->var.row_bytes;
  p->info.tile_n = p->var.bn;
  p->info.split = p->var.split;
  p->info.pair = p->var.pair == 1 ? 1 : 0;
  if (st == B200D2_OK && (flags & B200D2_PLAN_GRAPH)) {
    st = status_from_cuda(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    if (st == B200D2_OK) {
      const int st2 = plan_pipeline(p, p->stream, p->var);
      const cudaError_t e = cudaStreamEndCapture(p->stream, &p->graph);
      st = st2 != B200D2_OK ? st2 : status_from_cuda(e);
    }
    if (st == B200D2_OK) st = status_from_cuda(cudaGraphInstantiate(&p->exec, p->graph, 0));
    p->info.graph = (st == B200D2_OK) ? 1 : 0;
  }
  if (st != B200D2_OK) {
    plan_free(p);
    return st;
  }
  *out = p;
  return B200D2_OK;
}

extern "C" int b200d2_plan_run(b200d2_plan* p, void* stream) {
  if (!p) return B200D2_ERR_INVALID;
  b200d2::NvtxRange range("b200d2_plan_run");
  cudaStream_t s = (cudaStream_t)stream;
  if (p->exec) {
    B200D2_CUDA_TRY(cudaGraphLaunch(p->exec, s));
    b200d2::count_launch(b200d2::kNumStages);
    return B200D2_OK;
  }
  return b200d2::plan_pipeline(p, s, p->var);
}

extern "C" int b200d2_plan_get_info(const b200d2_plan* p, b200d2_plan_info* info) {
  if (!p || !info) return B200D2_ERR_INVALID;
  *info = p->info;
  return B200D2_OK;
}

extern "C" int b200d2_plan_destroy(b200d2_plan* p) {
  if (!p) return B200D2_ERR_INVALID;
  cudaStreamSynchronize(p->stream);
  b200d2::plan_free(p);
  return B200D2_OK;
}

// ------------------------------------------------------------------ merged batches
// Several requests on one reference in one pipeline run (the serving loop's
// merged admissions), block-diagonal: request r's particles are scored only
// against its own orientation columns [col0_r, col0_r + O_r) of the merged
// orientation set, at its own translations, through the uneven batch
// kernels (per-particle rows, orientation maps and outputs).  Unlike a plan,
// nothing is allocated, timed or synchronised: the tables are built on the
// host when the batch is created, and merged_enqueue copies them from the
// caller's page-locked staging area into the caller's device memory and
// launches the stages, all in the order of one stream.  The FP64 norms and
// the contraction run over work lists of the blocks some particle needs
// (particle tile x orientation tile, m tile x n tile), so no request pays
// for another's orientations there either.
namespace b200d2 {

struct MergedBatch {
  b200d2_view view;
  int prec = 0, N_img = 0, n = 0, P = 0, O = 0;
  std::vector<MergedRequest> req;
  std::vector<int> part0;          // first particle of each request
  std::vector<int4> rows;
  std::vector<int> row0;           // first row of each particle
  std::vector<int2> tiles[3];      // 128 x 256, 128 x 128, 256 x 256 (CTA pairs)
  std::vector<int2> ntile[3];      // norm kernel work lists (64-, 32-, 16-particle tiles)
  std::vector<float2> txy;
  std::vector<int> inv;            // [n][O]
  TcGeom g;
  GemmVariant var;
  // device layout from the caller's base: the workspace, then the tables
  // (mirrored byte for byte by the staging area)
  size_t off_tab = 0, off_parts = 0, off_rows = 0, off_tiles[3] = {0, 0, 0}, off_ntile[3] = {0, 0, 0}, off_txy = 0,
         off_inv = 0, dev_bytes = 0;
};

MergedBatch* merged_create(const b200d2_view& v, int N_img, int precision, const MergedRequest* r, int n, int O_cols,
                           int* status) {
  auto fail = [&](int st) -> MergedBatch* {
    if (status) *status = st;
    return nullptr;
  };
  if (!r || n <= 0 || N_img <= 0 || O_cols <= 0) return fail(B200D2_ERR_INVALID);
  if (!is_tc_precision(precision)) return fail(B200D2_ERR_UNSUPPORTED);
  if (v.mdlZ == 0 || (long long)v.imgX * v.imgY < N_img || v.maxR > 4096) return fail(B200D2_ERR_INVALID);
  for (int k = 0; k < n; ++k) {
    const MergedRequest& q = r[k];
    if (q.P <= 0 || q.O <= 0 || q.T <= 0 || !q.h_tx || !q.h_ty || q.col0 < 0 || q.col0 % 256 != 0 ||
        (long long)q.col0 + q.O > O_cols || (k > 0 && q.col0 < r[k - 1].col0 + r[k - 1].O))
      return fail(B200D2_ERR_INVALID);
    if ((long long)q.O * q.T >= 0xffffffffLL) return fail(B200D2_ERR_UNSUPPORTED);
  }
  MergedBatch* m = new MergedBatch();
  m->view = v;
  m->prec = precision;
  m->N_img = N_img;
  m->n = n;
  m->O = O_cols;
  m->req.assign(r, r + n);
  // translation sets shared between requests share their phase tables
  std::map<std::vector<std::pair<uint32_t, uint32_t>>, int> sets;
  std::vector<int> tab0(n), req_of;
  for (int k = 0; k < n; ++k) {
    const MergedRequest& q = r[k];
    std::vector<std::pair<uint32_t, uint32_t>> key(q.T);
    for (int t = 0; t < q.T; ++t) {
      uint32_t a, c;
      memcpy(&a, &q.h_tx[t], 4);
      memcpy(&c, &q.h_ty[t], 4);
      key[t] = {a, c};
    }
    auto it = sets.find(key);
    if (it == sets.end()) {
      it = sets.emplace(key, (int)m->txy.size()).first;
      for (int t = 0; t < q.T; ++t) m->txy.push_back(make_float2(q.h_tx[t], q.h_ty[t]));
    }
    tab0[k] = it->second;
    m->part0.push_back(m->P);
    for (int i = 0; i < q.P; ++i) {
      m->row0.push_back((int)m->rows.size());
      req_of.push_back(k);
      for (int t = 0; t < q.T; ++t) m->rows.push_back(make_int4(m->P + i, t, tab0[k] + t, 0));
    }
    m->P += q.P;
  }
  const int Mrows = (int)m->rows.size();
  const int Mtiles = (Mrows + 127) / 128, Ntiles = (O_cols + 255) / 256, Ntiles128 = (O_cols + 127) / 128;
  // work lists: an m tile's rows belong to a run of consecutive requests;
  // it needs the 128-column blocks of their column ranges
  auto blocks_of = [&](int rr0, int rr1, std::vector<char>& un) {
    std::fill(un.begin(), un.end(), 0);
    for (int k = req_of[m->rows[rr0].x]; k <= req_of[m->rows[rr1 - 1].x]; ++k)
      for (int c = r[k].col0 / 128; c <= (r[k].col0 + r[k].O - 1) / 128; ++c) un[c] = 1;
  };
  std::vector<char> un(Ntiles128, 0);
  for (int mt = 0; mt < (Mtiles + 1) / 2; ++mt) {  // 256-row m-tiles of CTA pairs
    blocks_of(mt * 256, std::min(Mrows, mt * 256 + 256), un);
    for (int c = 0; c < Ntiles; ++c)
      if (un[2 * c] || (2 * c + 1 < Ntiles128 && un[2 * c + 1])) m->tiles[2].push_back(make_int2(mt, c));
  }
  for (int mt = 0; mt < Mtiles; ++mt) {
    blocks_of(mt * 128, std::min(Mrows, mt * 128 + 128), un);
    for (int c = 0; c < Ntiles; ++c)
      if (un[2 * c] || (2 * c + 1 < Ntiles128 && un[2 * c + 1])) m->tiles[0].push_back(make_int2(mt, c));
    for (int c = 0; c < Ntiles128; ++c)
      if (un[c]) m->tiles[1].push_back(make_int2(mt, c));
  }
  // the norm kernel's blocks: a particle tile needs its requests' columns
  norma_lists(m->P, O_cols,
              [&](int pl, int blk) {
                const MergedRequest& q = r[req_of[pl]];
                return blk >= q.col0 / 128 && blk <= (q.col0 + q.O - 1) / 128;
              },
              m->ntile);
  m->inv.assign((size_t)n * O_cols, -1);
  for (int k = 0; k < n; ++k)
    for (int o = 0; o < r[k].O; ++o) m->inv[(size_t)k * O_cols + r[k].col0 + o] = o;

  b200d2_batch b;
  memset(&b, 0, sizeof(b));
  b.O = O_cols;
  b.T = (int)m->txy.size();  // number of phase tables
  b.P = m->P;
  b.N_img = N_img;
  b.img_stride = N_img;
  m->g = make_geom(v, b, precision, Mrows, false);
  // CTA pairs while their tiles give every pair of SMs one, else 128-wide
  // single-CTA tiles (twice the tiles); no k-splits
  if ((long long)m->tiles[2].size() >= num_sms() / 2) {
    m->var.row_bytes = 128;
    m->var.bn = 256;
    m->var.pair = 1;
  } else {
    m->var.row_bytes = gemm_row_bytes();
    m->var.bn = 128;
    m->var.pair = 2;
  }
  m->var.split = 1;
  size_t o = align_up(m->g.total, 256);
  m->off_tab = o;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align_up(o + bytes, 256);
    return at;
  };
  m->off_parts = take(sizeof(PartDev) * (size_t)m->P);
  m->off_rows = take(sizeof(int4) * m->rows.size());
  for (int w = 0; w < 3; ++w) m->off_tiles[w] = take(sizeof(int2) * std::max<size_t>(m->tiles[w].size(), 1));
  for (int w = 0; w < 3; ++w) m->off_ntile[w] = take(sizeof(int2) * std::max<size_t>(m->ntile[w].size(), 1));
  m->off_txy = take(sizeof(float2) * m->txy.size());
  m->off_inv = take(sizeof(int) * m->inv.size());
  m->dev_bytes = o;
  if (status) *status = B200D2_OK;
  return m;
}

size_t merged_device_bytes(const MergedBatch* m) { return m ? m->dev_bytes : 0; }
size_t merged_host_bytes(const MergedBatch* m) { return m ? m->dev_bytes - m->off_tab : 0; }
void merged_destroy(MergedBatch* m) { delete m; }

int merged_enqueue(MergedBatch* m, const float* d_eulers, const MergedDev* d, double* d_min, long long* d_argmin,
                   void* dmem, void* hstage, cudaStream_t s) {
  if (!m || !d_eulers || !d || !d_min || !d_argmin || !dmem || !hstage) return B200D2_ERR_INVALID;
  NvtxRange range("b200d2 merged batch");
  uint8_t* dev = static_cast<uint8_t*>(dmem);
  // the staging area mirrors the device tables: host(off) holds dev + off
  auto host = [&](size_t off) { return static_cast<uint8_t*>(hstage) + (off - m->off_tab); };
  const int* d_inv = reinterpret_cast<const int*>(dev + m->off_inv);
  PartDev* hp = reinterpret_cast<PartDev*>(host(m->off_parts));
  for (int k = 0; k < m->n; ++k) {
    const MergedRequest& q = m->req[k];
    if (!d[k].re || !d[k].im || !d[k].corr || !d[k].out) return B200D2_ERR_INVALID;
    for (int i = 0; i < q.P; ++i) {
      PartDev& x = hp[m->part0[k] + i];
      x.re = d[k].re + (size_t)i * m->N_img;
      x.im = d[k].im + (size_t)i * m->N_img;
      x.corr = d[k].corr + (size_t)i * m->N_img;
      x.out = d[k].out + (size_t)i * q.O * q.T;
      x.inv = d_inv + (size_t)k * m->O;
      x.T = q.T;
      x.O = q.O;
      x.row0 = m->row0[m->part0[k] + i];
      x.pad = 0;
    }
  }
  memcpy(host(m->off_rows), m->rows.data(), sizeof(int4) * m->rows.size());
  for (int w = 0; w < 3; ++w) memcpy(host(m->off_tiles[w]), m->tiles[w].data(), sizeof(int2) * m->tiles[w].size());
  for (int w = 0; w < 3; ++w) memcpy(host(m->off_ntile[w]), m->ntile[w].data(), sizeof(int2) * m->ntile[w].size());
  memcpy(host(m->off_txy), m->txy.data(), sizeof(float2) * m->txy.size());
  memcpy(host(m->off_inv), m->inv.data(), sizeof(int) * m->inv.size());
  B200D2_CUDA_TRY(cudaMemcpyAsync(dev + m->off_tab, hstage, m->dev_bytes - m->off_tab, cudaMemcpyHostToDevice, s));
  UnevenTabs U{reinterpret_cast<const PartDev*>(dev + m->off_parts),
               reinterpret_cast<const int4*>(dev + m->off_rows),
               {reinterpret_cast<const int2*>(dev + m->off_tiles[0]), reinterpret_cast<const int2*>(dev + m->off_tiles[1]),
                reinterpret_cast<const int2*>(dev + m->off_tiles[2])},
               {(int)m->tiles[0].size(), (int)m->tiles[1].size(), (int)m->tiles[2].size()},
               reinterpret_cast<const float2*>(dev + m->off_txy),
               (int)m->txy.size(),
               (int)m->rows.size(),
               {reinterpret_cast<const int2*>(dev + m->off_ntile[0]), reinterpret_cast<const int2*>(dev + m->off_ntile[1]),
                reinterpret_cast<const int2*>(dev + m->off_ntile[2])},
               {(int)m->ntile[0].size(), (int)m->ntile[1].size(), (int)m->ntile[2].size()},
               nullptr,
               -1};
  b200d2_batch b;
  memset(&b, 0, sizeof(b));
  b.d_eulers = d_eulers;
  b.O = m->O;
  b.T = (int)m->txy.size();
  b.P = m->P;
  b.N_img = m->N_img;
  b.d_real = d[0].re;  // unused by the tabled kernels; kept valid
  b.d_imag = d[0].im;
  b.d_corr = d[0].corr;
  b.img_stride = m->N_img;
  b.d_diff2 = d[0].out;
  b.d_min = d_min;
  b.d_argmin = d_argmin;
  int st = B200D2_OK;
  for (int i = 0; i < kNumStages && st == B200D2_OK; ++i) st = dispatch_stage(m->view, b, m->prec, m->g, dmem, i, s, &U, m->var);
  return st;
}

}  // namespace b200d2

// ------------------------------------------------------------------ kernel preload
// With CUDA's lazy module loading (the default), a kernel is loaded on its
// first launch, and loading it can wait for the work already running on the
// device.  A server whose requests pick tile shapes, norm tiles and
// contraction variants by size would meet new ones mid-run: one such load
// stalled every request in flight for about 30 ms at C5.  Loading every
// kernel a precision's pipeline can launch up front (cudaFuncGetAttributes
// loads the function) moves that cost to set-up.
namespace b200d2 {

template <int PREC>
static cudaError_t preload_prec() {
  cudaFuncAttributes a;
  cudaError_t e = cudaSuccess;
  auto get = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, f);
  };
  get((const void*)tc_project_kernel<PREC>);
  get((const void*)tc_project_scaled_kernel<PREC>);
  get((const void*)tc_gen_a_kernel<PREC, false>);
  get((const void*)tc_gen_a_kernel<PREC, true>);
  get((const void*)tc_gemm_kernel<PREC, 64, 128, false>);
  get((const void*)tc_gemm_kernel<PREC, 64, 256, false>);
  get((const void*)tc_gemm_kernel<PREC, 128, 128, false>);
  get((const void*)tc_gemm_kernel<PREC, 128, 256, false>);
  get((const void*)tc_gemm_kernel<PREC, 64, 128, true>);
  get((const void*)tc_gemm_kernel<PREC, 64, 256, true>);
  get((const void*)tc_gemm_kernel<PREC, 128, 128, true>);
  get((const void*)tc_gemm_kernel<PREC, 128, 256, true>);
  get((const void*)tc_gemm_pair_kernel<PREC, 64, false>);
  get((const void*)tc_gemm_pair_kernel<PREC, 128, false>);
  get((const void*)tc_gemm_pair_kernel<PREC, 64, true>);
  get((const void*)tc_gemm_pair_kernel<PREC, 128, true>);
  return e;
}

int tc_preload(int precision) {
  cudaFuncAttributes a;
  cudaError_t e = cudaSuccess;
  auto get = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, f);
  };
  get((const void*)tc_pixel_list_kernel);
  get((const void*)tc_phase_kernel);
  get((const void*)tc_phase2d_kernel);
  get((const void*)tc_phase_compact_kernel);
  get((const void*)tc_scale_a_kernel);
  get((const void*)tc_normx_kernel);
  get((const void*)tc_norma_kernel<4, 4, false>);
  get((const void*)tc_norma_kernel<2, 4, false>);
  get((const void*)tc_norma_kernel<1, 4, false>);
  get((const void*)tc_norma_kernel<1, 2, false>);
  get((const void*)tc_norma_kernel<1, 1, false>);
  get((const void*)tc_norma_kernel<4, 4, true>);
  get((const void*)tc_norma_kernel<2, 4, true>);
  get((const void*)tc_norma_kernel<1, 4, true>);
  get((const void*)tc_finalize_kernel);
  if (e != cudaSuccess) return status_from_cuda(e);
  switch (precision) {
    case B200D2_PREC_BF16X3: e = preload_prec<B200D2_PREC_BF16X3>(); break;
    case B200D2_PREC_TF32X3: e = preload_prec<B200D2_PREC_TF32X3>(); break;
    case B200D2_PREC_TF32: e = preload_prec<B200D2_PREC_TF32>(); break;
    case B200D2_PREC_FP16X3: e = preload_prec<B200D2_PREC_FP16X3>(); break;
    case B200D2_PREC_FP16: e = preload_prec<B200D2_PREC_FP16>(); break;
    default: return B200D2_ERR_UNSUPPORTED;
  }
  return status_from_cuda(e);
}

}  // namespace b200d2

extern "C" int b200d2_workspace_status(const void* d_workspace, void* stream, int* status) {
  if (!d_workspace || !status) return B200D2_ERR_INVALID;
  uint32_t v = 0;
  cudaStream_t s = (cudaStream_t)stream;
  B200D2_CUDA_TRY(cudaMemcpyAsync(&v, d_workspace, sizeof(v), cudaMemcpyDeviceToHost, s));
  B200D2_CUDA_TRY(cudaStreamSynchronize(s));
  *status = (int)v;
  return B200D2_OK;
}

extern "C" int b200d2_set_gemm_variant(int row_bytes, int tile_n, int split, int pair) {
  if ((row_bytes != 0 && row_bytes != 64 && row_bytes != 128) || (tile_n != 0 && tile_n != 128 && tile_n != 256) ||
      split < 0 || split > 64 || pair < 0 || pair > 2)
    return B200D2_ERR_INVALID;
  b200d2::g_var_rb.store(row_bytes);
  b200d2::g_var_bn.store(tile_n);
  b200d2::g_var_split.store(split);
  b200d2::g_var_pair.store(pair);
  return B200D2_OK;
}

extern "C" int b200d2_set_combine(int mode) {
  if (mode != B200D2_COMBINE_DF32 && mode != B200D2_COMBINE_FP64) return B200D2_ERR_INVALID;
  b200d2::g_combine64.store(mode == B200D2_COMBINE_FP64 ? 1 : 0);
  return B200D2_OK;
}

extern "C" int b200d2_set_wait_limit_ns(unsigned long long ns) {
  b200d2::g_wait_ns.store(ns);
  return B200D2_OK;
}

extern "C" int b200d2_set_operand_gen(int mode) {
  if (mode != 0 && mode != 1) return B200D2_ERR_INVALID;
  b200d2::g_operand_gen.store(mode);
  return B200D2_OK;
}

extern "C" int b200d2_set_batch_graphs(int enable) {
  if (enable != 0 && enable != 1) return B200D2_ERR_INVALID;
  b200d2::g_batch_graphs.store(enable);
  return B200D2_OK;
}
