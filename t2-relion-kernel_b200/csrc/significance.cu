// significance.cu -- significant coarse samples of a weighted batch
// (b200d2_significance).
//
// Reference: after the coarse weights, RELION's E-step (the pass-0 branch of
// convertAllSquaredDifferencesToWeights, not vendored in the reference
// harness) keeps the highest-weight samples that carry adaptive_fraction of a
// particle's weight.  Its device steps, per particle: drop the weights that
// are not > 0, sort the rest ascending, take inclusive cumulative sums c_k,
// find the index with cuda_kernel_find_threshold_idx_in_cumulative
// (src/cuda_device_utils.cuh:254-266: idx = i + 1 for the i with
// c_i <= thr < c_{i+1}, else 0) at thr = (1 - adaptive_fraction) * sum_weight,
// set nsig = count - idx, cap nsig at maximum_significants (idx = count -
// nsig), take the threshold weight sorted[idx], and mark w >= it with
// cuda_kernel_array_over_threshold (src/cuda_device_utils.cuh:238-252).
//
// Nothing is sorted in HBM.  Positive finite doubles order like their bit
// patterns read as unsigned integers (keys), so the threshold weight is found
// by narrowing a key range [klo, khi) that holds the crossing, keeping the
// exact count and sum of the weights below the range:
//
//  A. One pass over the weights.  Weights below 2^(ilogb(thr) - 64) (the
//     tail) weigh less than 2^-37 thr together and are only summed; the next
//     128 binades are counted (per-warp histograms in shared memory); above
//     them only a count and the smallest weight are kept.
//  K. A weight of binade e lies in [2^e, 2^(e+1)), so the counts bound the
//     cumulative sums within a factor of two: the range becomes the binades
//     from the first whose upper bound exceeds thr to the first whose lower
//     bound does (one to three binades in practice).
//  B. A second pass sums the weights between the tail and the range, writes
//     the mask of every weight outside it (1 above, 0 below) and compacts the
//     range's weights with their indices.
//  L. Levels over the candidates: count them in up to 8192 equal key
//     intervals, bound each interval's weight by count x its smallest and
//     largest value, narrow the range the same way, then sum the candidates
//     below the new range and compact those inside it.  Interval widths
//     shrink by 2^13 per level.
//  F. When at most 4096 candidates remain they are sorted in shared memory
//     and scanned exactly; when the intervals are single keys the exact sums
//     come from the counts, and ties are resolved by division.  Candidates
//     dropped above a range pass; the last ones are marked against the
//     threshold weight.
//
// Sums below the range are exact integers in units of 2^(ilogb(thr) - 100)
// (128-bit, added with atomics, so independent of the order of arrival);
// each thread first adds its weights with error-free two-sums in FP64 and
// converts once.  The result is that of exact cumulative sums, except where
// the crossing lies within about 2^-72 thr of a tie; a floating-point scan
// (the reference's) departs from exact sums far sooner.  Lists are cut into
// segments of 2048 weights, each written by one warp, so compaction needs no
// atomics.  The first level runs over all particles at once; deeper levels
// and the final step run in one CTA per particle, compacting in place.  Without a cap the weights are read twice and the mask written
// once; the levels touch only candidates.  With a cap the rank phase reruns
// the levels by counts from the whole array and writes those particles'
// masks in a full pass, as does a particle whose threshold weight is its
// smallest (thr at or above its total).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace b200d2 {
namespace {

using u64 = unsigned long long;

constexpr int kSThreads = 256;
constexpr int kWarps = kSThreads / 32;
constexpr long long kScanChunk = 16384;  // weights per CTA in passes A and B
constexpr int kSeg = 2048;               // list segment capacity (weights)
constexpr int kLevelCtas = 16;           // CTAs per particle in the passes over lists
constexpr int kWindow = 128;             // binades counted by pass A
constexpr int kBuckets = 8192;           // key intervals per level
constexpr int kSortMax = 4096;           // candidates sorted in shared memory
constexpr int kMaxLevels = 8;            // levels before a particle is reported unresolved
constexpr u64 kInfKey = 0x7FF0000000000000ull;
constexpr long long kMaxN = 1ll << 27;

enum : unsigned { kPhaseSum = 0, kPhaseRank = 1, kPhaseDone = 2 };
enum : unsigned { kStageLevel = 0, kStageLast = 1 };

struct SigState {
  u64 klo, khi;          // candidate key range
  u64 c_below;           // positive finite weights below klo
  u64 f_lo, f_hi;        // their sum (sum phase), 128-bit, units of 2^e_u
  u64 ncand;             // weights in [klo, khi)
  u64 rank;              // rank phase: target sorted position
  u64 npos;              // positive finite weights
  u64 tail_cnt, tail_u;  // pass A: tail count and sum (units)
  u64 above_cnt, above_maxnot, maxnot;  // pass A: above the window; ~key maxima
  u64 tail_key;          // tail limit 2^(ilogb(thr) - 64) as a key; 0: no tail
  double thr, sig;
  long long nsig;
  int e_u, e_lo, shift, last_level;  // unit exponent, window start, interval log2, level that ended the narrowing
  unsigned phase, stage, full_mask, pad;
};
static_assert(sizeof(SigState) == 168, "state layout");

// ---- 128-bit unsigned integers ---------------------------------------------
struct U128 {
  u64 lo, hi;
};
__device__ __forceinline__ U128 add128(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
  return r;
}
__device__ __forceinline__ U128 sub128(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo - b.lo;
  r.hi = a.hi - b.hi - (a.lo < b.lo ? 1ull : 0ull);
  return r;
}
__device__ __forceinline__ bool gt128(U128 a, U128 b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }
// a * q for q < 2^32 (no overflow for the values used here)
__device__ __forceinline__ U128 mul128(U128 a, u64 q) {
  U128 r;
  r.lo = a.lo * q;
  r.hi = __umul64hi(a.lo, q) + a.hi * q;
  return r;
}
// floor(v * 2^-e) for v >= 0, saturating at 2^104 (above any thr in units)
__device__ __forceinline__ U128 to_units(double v, int e) {
  const double x = ldexp(v, -e);
  if (!(x < 0x1p104)) return U128{0ull, 1ull << 40};
  const double h = trunc(ldexp(x, -64));
  const double r = __fma_rn(-h, 0x1p64, x);  // exact: x - h 2^64 lies in [0, 2^64)
  return U128{(u64)r, (u64)h};
}
// saturated value: above any partial sum compared with thr (< 2^102 units)
__device__ __forceinline__ U128 sat128() { return U128{0ull, 1ull << 40}; }
// v * cnt, saturating
__device__ __forceinline__ U128 mul_sat(U128 v, unsigned cnt) {
  if (v.hi >= (1ull << 40) || ((double)v.hi * 0x1p64 + (double)v.lo) * (double)cnt >= 0x1p103) return sat128();
  return mul128(v, cnt);
}
__device__ __forceinline__ double from_units(U128 a, int e) {
  return ldexp((double)a.hi, e + 64) + ldexp((double)a.lo, e);
}
__device__ __forceinline__ U128 shfl_up128(U128 a, int o) {
  return U128{__shfl_up_sync(0xffffffffu, a.lo, o), __shfl_up_sync(0xffffffffu, a.hi, o)};
}
__device__ __forceinline__ U128 warp_sum128(U128 a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    a = add128(a, U128{__shfl_xor_sync(0xffffffffu, a.lo, o), __shfl_xor_sync(0xffffffffu, a.hi, o)});
  return a;
}
// order-independent 128-bit global add
__device__ __forceinline__ void atomic_add128(u64* lo, u64* hi, U128 a) {
  const u64 old = atomicAdd(lo, a.lo);
  atomicAdd(hi, a.hi + (old + a.lo < old ? 1ull : 0ull));
}

// error-free FP64 accumulation of nonnegative weights
struct TwoSumAcc {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double w) {
    const double t = __dadd_rn(s, w);
    const double bb = __dsub_rn(t, s);
    c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, __dsub_rn(t, bb)), __dsub_rn(w, bb)));
    s = t;
  }
  // the total in units of 2^e (s is the rounded sum, c the remainder)
  __device__ __forceinline__ U128 units(int e) const {
    const U128 a = to_units(s, e);
    const U128 b = to_units(fabs(c), e);
    return c >= 0.0 ? add128(a, b) : sub128(a, b);
  }
};

__device__ __forceinline__ double key_value(u64 k) { return __longlong_as_double((long long)k); }
__device__ __forceinline__ u64 value_key(double v) { return (u64)__double_as_longlong(v); }

// kPerThread consecutive keys from index i (zero past hi); vec: 16-byte loads
constexpr int kPerThread = 8;
__device__ __forceinline__ void load_run(const u64* row, long long i, long long hi, bool vec,
                                         u64 (&kv)[kPerThread]) {
  if (vec && i + kPerThread - 1 < hi) {
#pragma unroll
    for (int h = 0; h < kPerThread / 2; ++h) {
      const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(row + i + 2 * h);
      kv[2 * h] = a.x;
      kv[2 * h + 1] = a.y;
    }
  } else {
#pragma unroll
    for (int u = 0; u < kPerThread; ++u) kv[u] = i + u < hi ? row[i + u] : 0ull;
  }
}

__device__ __forceinline__ int interval_shift(u64 span) {
  int sh = 0;
  while (sh < 63 && ((span - 1) >> sh) >= (u64)kBuckets) ++sh;
  return sh;
}

// Exclusive prefix of (a, c) over the CTA's threads in thread order, plus
// the block totals.  Uses two shared arrays of kWarps entries each.
__device__ __forceinline__ void block_scan128(U128 a, u64 c, U128& ex, u64& exc, u64* s_lo, u64* s_hi, u64* s_c) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  U128 inc = a;
  u64 ic = c;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const U128 o = shfl_up128(inc, off);
    const u64 oc = __shfl_up_sync(0xffffffffu, ic, off);
    if (lane >= off) {
      inc = add128(inc, o);
      ic += oc;
    }
  }
  __syncthreads();
  if (lane == 31) {
    s_lo[warp] = inc.lo;
    s_hi[warp] = inc.hi;
    s_c[warp] = ic;
  }
  __syncthreads();
  ex = sub128(inc, a);
  exc = ic - c;
  for (int w = 0; w < warp; ++w) {
    ex = add128(ex, U128{s_lo[w], s_hi[w]});
    exc += s_c[w];
  }
}

// ---- settling ---------------------------------------------------------------
// binned: the threshold weight came from the range that pass B compacted, so
// pass B and the scatter write this particle's mask; otherwise a full pass does.
__device__ void settle(SigState& S, unsigned phase, double v, long long nsig, long long maxsig, bool binned) {
  if (phase == kPhaseSum && maxsig > 0 && nsig > maxsig) {
    // cap: the threshold becomes the weight at sorted position npos - maxsig
    S.phase = kPhaseRank;
    S.stage = kStageLevel;
    S.rank = S.npos - (u64)maxsig;
    S.nsig = maxsig;
    S.klo = 1ull;
    S.khi = kInfKey;
    S.c_below = 0ull;
    S.ncand = S.npos;
    S.shift = interval_shift(kInfKey - 1ull);
    return;
  }
  S.sig = v;
  if (phase == kPhaseSum) S.nsig = nsig;
  S.full_mask = binned ? 0u : 1u;
  S.phase = kPhaseDone;
}

// idx = 0: the threshold weight is the smallest positive weight (or +inf when
// there is none, which only +inf weights pass)
__device__ void settle_smallest(SigState& S, long long maxsig) {
  if (S.npos == 0ull) {
    S.sig = key_value(kInfKey);
    S.nsig = 0;
    S.full_mask = 1u;
    S.phase = kPhaseDone;
  } else {
    settle(S, kPhaseSum, key_value(~S.maxnot), (long long)S.npos, maxsig, false);
  }
}

// ---- A: tail sum, window counts, above-window minimum -----------------------
// Thread t takes weights 8t..8t+7 of each group of 2048; consecutive weights
// of one binade are counted together.
__global__ void __launch_bounds__(kSThreads) sig_scan_kernel(const u64* __restrict__ keys, long long n, int vec,
                                                             const double* __restrict__ sum, double frac,
                                                             SigState* __restrict__ st, unsigned* __restrict__ gcnt) {
  const int p = blockIdx.y;
  SigState& S = st[p];
  const double thr = __dmul_rn(__dsub_rn(1.0, frac), sum[p]);
  const bool ok = thr > 0.0 && thr <= 1.7976931348623157e308;
  const int e = ok ? ilogb(thr) : 0;
  const u64 tail_key = ok ? value_key(ldexp(1.0, e - 64)) : 0ull;  // 0 below the subnormals
  const unsigned e_lo = ok ? (unsigned)max(0, e - 64 + 1023) : 0u;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.thr = thr;
    S.tail_key = tail_key;
    S.e_u = e - 100;
    S.e_lo = (int)e_lo;
  }
  __shared__ unsigned hc[kWarps][kWindow];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int b = lane; b < kWindow; b += 32) hc[warp][b] = 0u;
  __syncwarp();
  const unsigned tail_hi = (unsigned)(tail_key >> 32);  // a power of two: its low word is 0
  const long long lo = (long long)blockIdx.x * kScanChunk, hi = min(n, lo + kScanChunk);
  const u64* row = keys + (long long)p * n;
  double tsum = 0.0;
  u64 maxnot = 0ull;
  // above the window only the exponent of the smallest key is used later, so
  // the minimum of the keys' high words is kept (32-bit)
  unsigned amin_hi = 0xFFFFFFFFu;
  unsigned tcnt = 0u, acnt = 0u;
  for (long long i0 = lo; i0 < hi; i0 += kPerThread * kSThreads) {
    u64 kv[kPerThread];
    load_run(row, i0 + kPerThread * threadIdx.x, hi, vec, kv);
    unsigned run_b = 0u, run_n = 0u;
#pragma unroll
    for (int u = 0; u < kPerThread; ++u) {
      const u64 key = kv[u];
      const unsigned khw = (unsigned)(key >> 32);
      const bool pf = key != 0ull && khw < 0x7FF00000u;  // positive and finite
      const bool tail = pf && khw < tail_hi;
      const unsigned b = (khw >> 20) - e_lo;  // wraps below the window: tail weights
      const bool win = pf && !tail && b < (unsigned)kWindow;
      if (pf) maxnot = max(maxnot, ~key);
      if (tail) {
        tsum = __dadd_rn(tsum, key_value(key));
        ++tcnt;
      }
      if (pf && !tail && !win) {
        ++acnt;
        amin_hi = min(amin_hi, khw);
      }
      if (win) {
        if (run_n && b == run_b) {
          ++run_n;
        } else {
          if (run_n) atomicAdd(&hc[warp][run_b], run_n);
          run_b = b;
          run_n = 1u;
        }
      }
    }
    if (run_n) atomicAdd(&hc[warp][run_b], run_n);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    tsum = __dadd_rn(tsum, __shfl_xor_sync(0xffffffffu, tsum, o));
    tcnt += __shfl_xor_sync(0xffffffffu, tcnt, o);
    acnt += __shfl_xor_sync(0xffffffffu, acnt, o);
    maxnot = max(maxnot, __shfl_xor_sync(0xffffffffu, maxnot, o));
    amin_hi = min(amin_hi, __shfl_xor_sync(0xffffffffu, amin_hi, o));
  }
  if (lane == 0) {
    if (tcnt) {
      // the tail is below 2^-37 thr (< 2^63 units), so FP64 rounding here is
      // below 2^-89 thr
      atomicAdd(&S.tail_cnt, (u64)tcnt);
      atomicAdd(&S.tail_u, to_units(tsum, e - 100).lo);
    }
    if (acnt) {
      atomicAdd(&S.above_cnt, (u64)acnt);
      atomicMax(&S.above_maxnot, ~((u64)amin_hi << 32));  // (~above_maxnot) >> 52: that key's exponent
    }
    if (maxnot) atomicMax(&S.maxnot, maxnot);
  }
  __syncthreads();
  unsigned* gp = gcnt + (long long)p * kBuckets;
  for (int b = threadIdx.x; b < kWindow && (int)e_lo + b < 2048; b += kSThreads) {
    unsigned c = 0u;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) c += hc[w][b];
    if (c) atomicAdd(&gp[b], c);
  }
}

// ---- K: the range of binades, one warp per particle -------------------------
// Plain FP64 bound sums with a 2^-40 margin (their rounding is below 2^-45).
__global__ void __launch_bounds__(128) sig_bracket_kernel(SigState* __restrict__ st, int P,
                                                           unsigned* __restrict__ gcnt, long long maxsig) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (p >= P) return;
  SigState& S = st[p];
  const int e_lo = S.e_lo;
  unsigned* cn = gcnt + (long long)p * kBuckets;
  unsigned c[4];
  double lw = 0.0, uw = 0.0;
  u64 lc = 0ull;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int b = 4 * lane + k, E = e_lo + b;
    c[k] = E < 2048 ? cn[b] : 0u;
    cn[b] = 0u;
    if (c[k]) {
      lc += c[k];
      lw += E ? ldexp((double)c[k], E - 1023) : 0.0;
      uw += ldexp((double)c[k], (E ? E : 1) + 1 - 1023);
    }
  }
  double li = lw, ui = uw;
  u64 ci = lc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double ol = __shfl_up_sync(0xffffffffu, li, off), ou = __shfl_up_sync(0xffffffffu, ui, off);
    const u64 oc = __shfl_up_sync(0xffffffffu, ci, off);
    if (lane >= off) {
      li += ol;
      ui += ou;
      ci += oc;
    }
  }
  const u64 win_total = __shfl_sync(0xffffffffu, ci, 31);
  const double thr = S.thr;
  const double tail = ldexp((double)S.tail_u, S.e_u);
  const double tail_up = ldexp((double)S.tail_u + (double)S.tail_cnt, S.e_u);
  double lex = __shfl_up_sync(0xffffffffu, li, 1), uex = __shfl_up_sync(0xffffffffu, ui, 1);
  u64 cex = __shfl_up_sync(0xffffffffu, ci, 1);
  if (lane == 0) {
    lex = uex = 0.0;
    cex = 0ull;
  }
  const double up = 1.0 + 0x1p-40, dn = 1.0 - 0x1p-40;
  int blo = -1, bhi = -1, blast = -1;
  u64 cblo = 0ull;
  double L = tail + lex, U = tail_up + uex;
  u64 cw = cex;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!c[k]) continue;
    const int E = e_lo + 4 * lane + k;
    blast = E;
    L += E ? ldexp((double)c[k], E - 1023) : 0.0;
    U += ldexp((double)c[k], (E ? E : 1) + 1 - 1023);
    if (blo < 0 && U * up > thr) {
      blo = E;
      cblo = cw;  // window weights below binade E
    }
    if (bhi < 0 && L * dn > thr) bhi = E;
    cw += c[k];
  }
  const unsigned mlo = __ballot_sync(0xffffffffu, blo >= 0);
  const unsigned mhi = __ballot_sync(0xffffffffu, bhi >= 0);
  const unsigned mla = __ballot_sync(0xffffffffu, blast >= 0);
  const int slo = mlo ? __ffs(mlo) - 1 : 0;
  const int br_lo = mlo ? __shfl_sync(0xffffffffu, blo, slo) : -1;
  const u64 c_lo = __shfl_sync(0xffffffffu, cblo, slo);
  const int br_hi = mhi ? __shfl_sync(0xffffffffu, bhi, __ffs(mhi) - 1) : -1;
  const int last = mla ? __shfl_sync(0xffffffffu, blast, 31 - __clz(mla)) : -1;
  if (lane != 0) return;
  S.npos = S.tail_cnt + win_total + S.above_cnt;
  if (!(thr > 0.0 && thr <= 1.7976931348623157e308)) {
    settle_smallest(S, maxsig);  // no c_i <= thr < c_{i+1} (or thr < c_0): idx = 0
    return;
  }
  const int amin = S.above_cnt ? (int)((~S.above_maxnot) >> 52) : -1;
  int r_lo, r_hi;
  u64 below;
  if (br_lo < 0) {
    if (amin < 0) {  // the whole weight stays at or below thr: idx = 0
      settle_smallest(S, maxsig);
      return;
    }
    // the window stays at or below thr; the smallest weight above it exceeds
    // thr alone, so its binade holds the crossing
    r_lo = r_hi = amin;
    below = win_total;
  } else {
    r_lo = br_lo;
    r_hi = br_hi >= 0 ? br_hi : (amin >= 0 ? amin : last);
    below = c_lo;
  }
  S.klo = max((u64)r_lo << 52, S.tail_key);
  S.khi = (u64)(r_hi + 1) << 52;
  S.c_below = S.tail_cnt + below;
  S.f_lo = S.tail_u;
  S.f_hi = 0ull;
  S.shift = interval_shift(S.khi - S.klo);
  S.stage = kStageLevel;
}

// Candidate segment s of particle p: a list segment, or (whole) 2048
// consecutive weights of the array.
struct SegView {
  const u64* k;
  unsigned len;
};
__device__ __forceinline__ SegView seg_view(const u64* keys, const u64* list, const unsigned* segc, int p, int s,
                                            long long n, long long cap, int nseg, bool whole) {
  if (whole) {
    const long long b = (long long)s * kSeg;
    return {keys + (long long)p * n + b, (unsigned)max(0ll, min((long long)kSeg, n - b))};
  }
  return {list + (long long)p * cap + (long long)s * kSeg, segc[(long long)p * nseg + s]};
}

// ---- B: sum between the tail and the range, mask outside it, compaction -----
// Thread t takes weights 8t..8t+7 of each group of 2048, so warp w of CTA c
// covers 2048 weights of the chunk and writes root-list segment 8c + w
// (keys, indices, count).  The range's weights are also counted in its
// first-level key intervals.  vec: 16-byte loads; vmask: 8-byte mask stores.
__global__ void __launch_bounds__(kSThreads) sig_bin_kernel(const u64* __restrict__ keys, long long n, int vec,
                                                            int vmask, long long cap, int nseg,
                                                            SigState* __restrict__ st, u64* __restrict__ rk,
                                                            unsigned* __restrict__ ri, unsigned* __restrict__ rc,
                                                            unsigned* __restrict__ gcnt, uint8_t* __restrict__ passed) {
  const int p = blockIdx.y;
  SigState& S = st[p];
  if (S.phase != kPhaseSum) return;
  const u64 low_min = max(S.tail_key, 1ull), klo = S.klo, khi = S.khi;
  const int sh = S.shift;
  __shared__ unsigned hc[kBuckets];
  for (int b = threadIdx.x; b < kBuckets; b += kSThreads) hc[b] = 0u;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long lo = (long long)blockIdx.x * kScanChunk, hi = min(n, lo + kScanChunk);
  const u64* row = keys + (long long)p * n;
  const int seg = blockIdx.x * kWarps + warp;
  u64* ok = rk + (long long)p * cap + (long long)seg * kSeg;
  unsigned* oi = ri + (long long)p * cap + (long long)seg * kSeg;
  uint8_t* out = passed ? passed + (long long)p * n : nullptr;
  TwoSumAcc acc;
  unsigned cnt = 0u;  // warp-uniform
  for (long long i0 = lo; i0 < hi; i0 += kPerThread * kSThreads) {
    const long long i = i0 + kPerThread * threadIdx.x;
    u64 kv[kPerThread];
    load_run(row, i, hi, vec, kv);
    u64 mword = 0ull;
#pragma unroll
    for (int u = 0; u < kPerThread; ++u) {
      const u64 key = kv[u];
      // above the range: passes (+inf included); below it, zeros, negatives
      // and NaN fail; the range's own bits are written by the later steps
      if (key >= khi && key <= kInfKey) mword |= 1ull << (8 * u);
      if (key >= low_min && key < klo) acc.add(key_value(key));
      const bool in = key >= klo && key < khi;
      if (in) atomicAdd(&hc[(unsigned)((key - klo) >> sh)], 1u);
      const unsigned bal = __ballot_sync(0xffffffffu, in);
      if (in) {
        const unsigned at = cnt + __popc(bal & ((1u << lane) - 1u));
        ok[at] = key;
        oi[at] = (unsigned)(i + u);
      }
      cnt += __popc(bal);
    }
    if (out) {
      if (vmask && i + kPerThread - 1 < hi) {
        *reinterpret_cast<u64*>(out + i) = mword;
      } else {
#pragma unroll
        for (int u = 0; u < kPerThread; ++u)
          if (i + u < hi) out[i + u] = (uint8_t)((mword >> (8 * u)) & 1ull);
      }
    }
  }
  if (lane == 0) rc[(long long)p * nseg + seg] = cnt;
  const U128 sm = warp_sum128(acc.units(S.e_u));
  if (lane == 0 && (sm.lo | sm.hi)) atomic_add128(&S.f_lo, &S.f_hi, sm);
  __syncthreads();
  unsigned* gp = gcnt + (long long)p * kBuckets;
  for (int b = threadIdx.x; b < kBuckets; b += kSThreads)
    if (hc[b]) atomicAdd(&gp[b], hc[b]);
}

// ---- rank phase, first level: counts over the whole array ------------------
__global__ void __launch_bounds__(kSThreads) sig_count_kernel(const u64* __restrict__ keys, long long n,
                                                              SigState* __restrict__ st, unsigned* __restrict__ gcnt) {
  const int p = blockIdx.y;
  const SigState& S = st[p];
  if (S.phase != kPhaseRank || S.stage != kStageLevel) return;
  const u64 klo = S.klo, khi = S.khi;
  const int sh = S.shift;
  __shared__ unsigned hc[kBuckets];
  for (int b = threadIdx.x; b < kBuckets; b += kSThreads) hc[b] = 0u;
  __syncthreads();
  const long long lo = (long long)blockIdx.x * kScanChunk, hi = min(n, lo + kScanChunk);
  const u64* row = keys + (long long)p * n;
  for (long long i = lo + threadIdx.x; i < hi; i += kSThreads) {
    const u64 key = row[i];
    if (key >= klo && key < khi) atomicAdd(&hc[(unsigned)((key - klo) >> sh)], 1u);
  }
  __syncthreads();
  unsigned* gp = gcnt + (long long)p * kBuckets;
  for (int b = threadIdx.x; b < kBuckets; b += kSThreads)
    if (hc[b]) atomicAdd(&gp[b], hc[b]);
}

// ---- narrowing: one CTA per particle, all threads ---------------------------
// Thread t holds the counts of intervals [32t, 32t + 32) in c.  Sum phase:
// interval b holds cnt_b weights in [v(start_b), v(end_b)), so the cumulative
// sum through it lies between F + sum cnt v(start) and F + sum cnt v(end); the
// new range runs from the first interval whose upper bound exceeds thr to the
// first whose lower bound does (FP64 bound sums with a 2^-40 margin).  Rank
// phase: the interval holding the target position.  When every interval is a
// single key the sums are exact and the particle settles here.  S is written
// by thread 0; the function ends with a barrier.
constexpr int kPer = kBuckets / kSThreads;  // 32

__device__ void narrow_step(SigState& S, const unsigned (&c)[kPer], int level, unsigned phase, long long maxsig) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool sum_mode = phase == kPhaseSum;
  const u64 klo = S.klo, khi = S.khi;
  const int sh = S.shift;
  const int e_u = S.e_u;
  const double thr = S.thr;
  const u64 rank = S.rank, c_below = S.c_below;
  const U128 F = U128{S.f_lo, S.f_hi};
  auto start = [&](int b) { return klo + ((u64)b << sh); };
  auto end = [&](int b) { return min(khi, klo + ((u64)(b + 1) << sh)); };
  __shared__ u64 x_lo[kWarps], x_hi[kWarps], x_c[kWarps];
  __shared__ double x_l[kWarps], x_u[kWarps];
  __shared__ int s_blo, s_bhi, s_last;
  __shared__ u64 s_cblo, s_cin, s_plo, s_phi;
  __shared__ unsigned s_pcnt;
  if (tid == 0) {
    s_blo = s_bhi = kBuckets;
    s_last = -1;
    s_cin = 0ull;
  }

  if (sh == 0) {
    // every interval is a single key: exact cumulative sums (sum phase) or
    // counts (rank phase)
    U128 part = {0ull, 0ull};
    u64 pc = 0ull;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      if (!c[k]) continue;
      pc += c[k];
      if (sum_mode) part = add128(part, mul_sat(to_units(key_value(start(tid * kPer + k)), e_u), c[k]));
    }
    U128 ex;
    u64 exc;
    block_scan128(part, pc, ex, exc, x_lo, x_hi, x_c);
    const U128 thr_u = to_units(thr, e_u);
    U128 run = add128(F, ex);
    u64 C = c_below + exc;
    int pick = -1;
    unsigned pcnt = 0u;
    U128 before = run;
    u64 cb = C;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      if (!c[k] || pick >= 0) continue;
      const U128 nrun = sum_mode ? add128(run, mul_sat(to_units(key_value(start(tid * kPer + k)), e_u), c[k])) : run;
      if (sum_mode ? gt128(nrun, thr_u) : (C + c[k] > rank)) {
        pick = tid * kPer + k;
        pcnt = c[k];
        before = run;
        cb = C;
      }
      run = nrun;
      C += c[k];
    }
    if (pick >= 0) atomicMin(&s_blo, pick);
    __syncthreads();
    if (pick >= 0 && pick == s_blo) {
      s_plo = before.lo;
      s_phi = before.hi;
      s_cblo = cb;
      s_pcnt = pcnt;
    }
    __syncthreads();
    if (tid == 0) {
      if (s_blo == kBuckets) {  // no key exceeds thr: no crossing
        settle_smallest(S, maxsig);
      } else {
        const double v = key_value(start(s_blo));
        if (!sum_mode) {
          settle(S, phase, v, S.nsig, maxsig, false);
        } else {
          // ties at the key: the first of them whose inclusive sum exceeds
          // thr is at position q = floor((thr - before) / v) among them
          const U128 D = sub128(thr_u, U128{s_plo, s_phi});
          const U128 V = to_units(v, e_u);
          const u64 m = s_pcnt;
          const double qd = floor(from_units(D, 0) / from_units(V, 0));
          u64 q = qd < 0.0 ? 0ull : (qd > (double)m ? m : (u64)qd);
          while (q + 1 < m && !gt128(mul128(V, q + 1), D)) ++q;
          while (q > 0 && gt128(mul128(V, q), D)) --q;
          settle(S, phase, v, (long long)(S.npos - (s_cblo + q)), maxsig, true);
        }
      }
    }
    __syncthreads();
    return;
  }

  double lw = 0.0, uw = 0.0;
  u64 lc = 0ull;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    if (!c[k]) continue;
    const int b = tid * kPer + k;
    lc += c[k];
    if (sum_mode) {
      lw += (double)c[k] * key_value(start(b));
      uw += (double)c[k] * key_value(end(b));
    }
  }
  // block scan of (lw, uw, lc): within warps, then the warp totals in order
  double li = lw, ui = uw;
  u64 ci = lc;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double ol = __shfl_up_sync(0xffffffffu, li, off), ou = __shfl_up_sync(0xffffffffu, ui, off);
    const u64 oc = __shfl_up_sync(0xffffffffu, ci, off);
    if (lane >= off) {
      li += ol;
      ui += ou;
      ci += oc;
    }
  }
  if (lane == 31) {
    x_l[warp] = li;
    x_u[warp] = ui;
    x_c[warp] = ci;
  }
  __syncthreads();
  const double F0 = sum_mode ? from_units(F, e_u) : 0.0;
  double L = F0, U = F0;
  u64 C = c_below;
  for (int w = 0; w < warp; ++w) {
    L += x_l[w];
    U += x_u[w];
    C += x_c[w];
  }
  L += li - lw;
  U += ui - uw;
  C += ci - lc;
  const double up = 1.0 + 0x1p-40, dn = 1.0 - 0x1p-40;
  int blo = -1, bhi = -1, blast = -1;
  u64 cblo = 0ull;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    if (!c[k]) continue;
    const int b = tid * kPer + k;
    blast = b;
    const u64 nC = C + c[k];
    if (sum_mode) {
      L += (double)c[k] * key_value(start(b));
      U += (double)c[k] * key_value(end(b));
      if (blo < 0 && U * up > thr) {
        blo = b;
        cblo = C;
      }
      if (bhi < 0 && L * dn > thr) bhi = b;
    } else if (blo < 0 && nC > rank) {
      blo = bhi = b;
      cblo = C;
    }
    C = nC;
  }
  if (blo >= 0) atomicMin(&s_blo, blo);
  if (bhi >= 0) atomicMin(&s_bhi, bhi);
  if (blast >= 0) atomicMax(&s_last, blast);
  __syncthreads();
  if (blo >= 0 && blo == s_blo) s_cblo = cblo;
  const int b_lo = s_blo, b_hi = s_bhi < kBuckets ? s_bhi : s_last;
  // exact count of the candidates in the new range
  u64 in = 0ull;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int b = tid * kPer + k;
    if (b >= b_lo && b <= b_hi) in += c[k];
  }
  if (in) atomicAdd(&s_cin, in);
  __syncthreads();
  if (tid == 0) {
    if (b_lo == kBuckets) {
      // no interval exceeds thr even at its upper bound: no crossing at all
      settle_smallest(S, maxsig);
    } else {
      const u64 nlo = start(b_lo), nhi = end(b_hi);
      S.klo = nlo;
      S.khi = nhi;
      S.c_below = s_cblo;
      S.ncand = s_cin;
      S.shift = interval_shift(nhi - nlo);
      if (s_cin <= (u64)kSortMax) {
        S.stage = kStageLast;  // compacted once more, then sorted
        S.last_level = level;
      }
    }
  }
  __syncthreads();
}

// first level: the histogram is in global memory (cleared as it is read)
__global__ void __launch_bounds__(kSThreads) sig_narrow_kernel(unsigned phase, SigState* __restrict__ st,
                                                               unsigned* __restrict__ gcnt, long long maxsig) {
  const int p = blockIdx.x;
  SigState& S = st[p];
  if (S.phase != phase || S.stage != kStageLevel) return;
  unsigned* gp = gcnt + (long long)p * kBuckets + threadIdx.x * kPer;
  unsigned c[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    c[k] = gp[k];
    gp[k] = 0u;
  }
  narrow_step(S, c, 0, phase, maxsig);
}

// ---- first level: sum the candidates below the new range, compact those in it
// Input segment s (root list, or 2048 weights of the array in the rank phase)
// maps to segment s of the level list; every level-list segment's count is
// written.  Sum phase: candidates above the new range pass (mask 1 through
// their indices); the level list keeps the indices of the others.
__global__ void __launch_bounds__(kSThreads) sig_level_kernel(const u64* __restrict__ keys, const u64* __restrict__ rk,
                                                              const unsigned* __restrict__ ri,
                                                              const unsigned* __restrict__ rc, u64* __restrict__ lk,
                                                              unsigned* __restrict__ li, unsigned* __restrict__ lc,
                                                              long long n, long long cap, int nseg, unsigned phase,
                                                              SigState* __restrict__ st, uint8_t* __restrict__ passed) {
  const int p = blockIdx.y;
  SigState& S = st[p];
  if (S.phase != phase || !(S.stage == kStageLevel || S.last_level == 0)) return;
  const bool whole = phase == kPhaseRank;
  const int nsegs = whole ? (int)((n + kSeg - 1) / kSeg) : nseg;
  const u64 klo = S.klo, khi = S.khi;
  const bool sum_mode = phase == kPhaseSum;
  uint8_t* out = sum_mode && passed ? passed + (long long)p * n : nullptr;
  const int lane = threadIdx.x & 31, gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
  TwoSumAcc acc;
  for (int s = gw; s < nseg; s += gridDim.x * kWarps) {
    unsigned cnt = 0u;  // warp-uniform
    if (s < nsegs) {
      const SegView v = seg_view(keys, rk, rc, p, s, n, cap, nseg, whole);
      const unsigned* ix = ri + (long long)p * cap + (long long)s * kSeg;
      u64* o = lk + (long long)p * cap + (long long)s * kSeg;
      unsigned* oi = li + (long long)p * cap + (long long)s * kSeg;
      for (unsigned j0 = 0; j0 < v.len; j0 += 128) {  // four groups of 32 loaded together
        u64 kk[4];
        unsigned xx[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const unsigned j = j0 + 32 * u + lane;
          kk[u] = j < v.len ? v.k[j] : 0ull;
          xx[u] = (sum_mode && j < v.len) ? ix[j] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const u64 key = kk[u];
          if (sum_mode && key != 0ull && key < klo) acc.add(key_value(key));
          const bool in = key >= klo && key < khi;
          if (out && key >= khi && j0 + 32 * u + lane < v.len) out[xx[u]] = 1;
          const unsigned bal = __ballot_sync(0xffffffffu, in);
          if (in) {
            const unsigned at = cnt + __popc(bal & ((1u << lane) - 1u));
            o[at] = key;
            if (sum_mode) oi[at] = xx[u];
          }
          cnt += __popc(bal);
        }
      }
    }
    if (lane == 0) lc[(long long)p * nseg + s] = cnt;
  }
  if (sum_mode) {
    const U128 sm = warp_sum128(acc.units(S.e_u));
    if (lane == 0 && (sm.lo | sm.hi)) atomic_add128(&S.f_lo, &S.f_hi, sm);
  }
}

// ---- deeper levels and the final step: one CTA per particle ------------------
// Levels 1.. count, narrow and compact the level list in place (a warp reads
// each group of 32 keys before writing any of it, and writes only at or below
// what it has read).  With at most 4096 candidates left they are sorted in
// shared memory and scanned exactly.
__global__ void __launch_bounds__(kSThreads) sig_deep_kernel(u64* __restrict__ lk, unsigned* __restrict__ li,
                                                             unsigned* __restrict__ lc, long long n, long long cap,
                                                             int nseg, unsigned phase, SigState* __restrict__ st,
                                                             long long maxsig, uint8_t* __restrict__ passed) {
  constexpr int kSortPer = kSortMax / kSThreads;  // 16
  const int p = blockIdx.x;
  SigState& S = st[p];
  if (S.phase != phase) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool sum_mode = phase == kPhaseSum;
  u64* klist = lk + (long long)p * cap;
  unsigned* ilist = li + (long long)p * cap;
  unsigned* kcnt = lc + (long long)p * nseg;
  uint8_t* out = sum_mode && passed ? passed + (long long)p * n : nullptr;
  // mask bits of the current list once the threshold weight is known
  auto scatter_list = [&](u64 sk) {
    if (!out) return;
    for (int s = warp; s < nseg; s += kWarps) {
      const unsigned len = kcnt[s];
      const u64* k = klist + (long long)s * kSeg;
      const unsigned* ix = ilist + (long long)s * kSeg;
      for (unsigned j = lane; j < len; j += 32) out[ix[j]] = k[j] >= sk ? 1 : 0;
    }
  };
  __shared__ u64 buf[kSortMax];  // the level histogram, then the sorted candidates
  unsigned* hc = reinterpret_cast<unsigned*>(buf);
  static_assert(kBuckets * sizeof(unsigned) == kSortMax * sizeof(u64), "shared buffer");

  for (int level = 1; level < kMaxLevels && S.phase == phase && S.stage == kStageLevel; ++level) {
    const u64 klo = S.klo, khi = S.khi;
    const int sh = S.shift;
    for (int b = tid; b < kBuckets; b += kSThreads) hc[b] = 0u;
    __syncthreads();
    for (int s = warp; s < nseg; s += kWarps) {
      const unsigned len = kcnt[s];
      const u64* k = klist + (long long)s * kSeg;
      for (unsigned j = lane; j < len; j += 32) {
        const u64 key = k[j];
        if (key >= klo && key < khi) atomicAdd(&hc[(unsigned)((key - klo) >> sh)], 1u);
      }
    }
    __syncthreads();
    unsigned c[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) c[k] = hc[tid * kPer + k];
    __syncthreads();
    narrow_step(S, c, level, phase, maxsig);
    if (S.phase != phase) {  // settled (or sent to the rank phase)
      if (S.phase == kPhaseDone && !S.full_mask) scatter_list(value_key(S.sig));
      break;
    }
    // sum below the new range, compact in place
    const u64 nlo = S.klo, nhi = S.khi;
    TwoSumAcc acc;
    for (int s = warp; s < nseg; s += kWarps) {
      const unsigned len = kcnt[s];
      u64* k = klist + (long long)s * kSeg;
      unsigned cnt = 0u;
      unsigned* ix = ilist + (long long)s * kSeg;
      for (unsigned j0 = 0; j0 < len; j0 += 32) {
        const unsigned j = j0 + lane;
        const u64 key = j < len ? k[j] : 0ull;
        const unsigned idx = (sum_mode && j < len) ? ix[j] : 0u;
        if (sum_mode && key != 0ull && key < nlo) acc.add(key_value(key));
        const bool in = key >= nlo && key < nhi;
        if (out && j < len && key >= nhi) out[idx] = 1;
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (in) {
          const unsigned at = cnt + __popc(bal & ((1u << lane) - 1u));
          k[at] = key;
          if (sum_mode) ix[at] = idx;
        }
        cnt += __popc(bal);
      }
      __syncwarp();
      if (lane == 0) kcnt[s] = cnt;
    }
    if (sum_mode) {
      const U128 sm = warp_sum128(acc.units(S.e_u));
      U128 ex;
      u64 exc;
      __shared__ u64 d_lo[kWarps], d_hi[kWarps], d_c[kWarps];
      block_scan128(lane == 0 ? sm : U128{0ull, 0ull}, 0ull, ex, exc, d_lo, d_hi, d_c);
      if (tid == kSThreads - 1) {  // the block total: exclusive prefix of the last thread plus its value
        const U128 tot = add128(ex, lane == 0 ? sm : U128{0ull, 0ull});
        const U128 f = add128(U128{S.f_lo, S.f_hi}, tot);
        S.f_lo = f.lo;
        S.f_hi = f.hi;
      }
    }
    __syncthreads();
  }
  if (S.phase != phase) return;
  if (S.stage != kStageLast || S.ncand > (u64)kSortMax) {
    // not narrowed to a sortable set within kMaxLevels levels (never seen):
    // reported as nsig = -1 with a NaN threshold, which no weight passes
    if (tid == 0) {
      S.sig = __longlong_as_double(0x7FF8000000000000ll);
      S.nsig = -1;
      S.full_mask = 1u;
      S.phase = kPhaseDone;
    }
    return;
  }

  // gather the candidates (at most 4096) from the segments
  const u64 ncand = S.ncand, c_below = S.c_below;
  unsigned my = 0u;
  for (int s = tid; s < nseg; s += kSThreads) my += kcnt[s];
  unsigned inc = my;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned o = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += o;
  }
  __shared__ unsigned s_w[kWarps];
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  unsigned base = inc - my;
  for (int w = 0; w < warp; ++w) base += s_w[w];
  for (int s = tid; s < nseg; s += kSThreads) {
    const unsigned len = kcnt[s];
    const u64* src = klist + (long long)s * kSeg;
    for (unsigned j = 0; j < len && base + j < (unsigned)kSortMax; ++j) buf[base + j] = src[j];
    base += len;
  }
  const unsigned m = (unsigned)ncand;
  unsigned n2 = 1u;
  while (n2 < m) n2 <<= 1;
  for (unsigned j = m + tid; j < n2; j += kSThreads) buf[j] = ~0ull;
  __syncthreads();
  // bitonic sort, ascending
  for (unsigned k = 2; k <= n2; k <<= 1) {
    for (unsigned j = k >> 1; j > 0; j >>= 1) {
      for (unsigned i = tid; i < n2; i += kSThreads) {
        const unsigned l = i ^ j;
        if (l > i) {
          const u64 a = buf[i], b = buf[l];
          if ((a > b) == ((i & k) == 0)) {
            buf[i] = b;
            buf[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  if (!sum_mode) {
    if (tid == 0) settle(S, phase, key_value(buf[min(S.rank - c_below, (u64)m - 1)]), S.nsig, maxsig, false);
    return;
  }
  // exact inclusive prefix sums in sorted order: thread t holds [16t, 16t+16)
  const int e_u = S.e_u;
  U128 part = {0ull, 0ull};
#pragma unroll
  for (int k = 0; k < kSortPer; ++k) {
    const unsigned i = tid * kSortPer + k;
    if (i < m) part = add128(part, to_units(key_value(buf[i]), e_u));
  }
  U128 ex;
  u64 exc;
  __shared__ u64 f_lo[kWarps], f_hi[kWarps], f_c[kWarps];
  block_scan128(part, 0ull, ex, exc, f_lo, f_hi, f_c);
  __shared__ int s_pick;
  if (tid == 0) s_pick = kSortMax;
  __syncthreads();
  const U128 thr_u = to_units(S.thr, e_u);  // exact: thr is a multiple of 2^e_u
  U128 run = add128(U128{S.f_lo, S.f_hi}, ex);
  int pick = -1;
#pragma unroll
  for (int k = 0; k < kSortPer; ++k) {
    const unsigned i = tid * kSortPer + k;
    if (i < m && pick < 0) {
      run = add128(run, to_units(key_value(buf[i]), e_u));
      if (gt128(run, thr_u)) pick = (int)i;
    }
  }
  if (pick >= 0) atomicMin(&s_pick, pick);
  __syncthreads();
  const int pk = s_pick;
  const u64 sk = pk < kSortMax ? buf[pk] : 0ull;
  __syncthreads();
  if (tid == 0) {
    if (pk == kSortMax)  // every candidate stays at or below thr: no crossing
      settle_smallest(S, maxsig);
    else
      settle(S, phase, key_value(sk), (long long)(S.npos - (c_below + (u64)pk)), maxsig, true);
  }
  __syncthreads();
  if (S.phase == kPhaseDone && !S.full_mask) scatter_list(sk);
}

// ---- full-pass masks -------------------------------------------------------
__global__ void __launch_bounds__(kSThreads) sig_fullmask_kernel(const double* __restrict__ w, long long n,
                                                                 const SigState* __restrict__ st,
                                                                 uint8_t* __restrict__ passed) {
  const int p = blockIdx.y;
  if (!st[p].full_mask) return;
  const double sig = st[p].sig;
  const long long lo = (long long)blockIdx.x * kScanChunk, hi = min(n, lo + kScanChunk);
  const double* row = w + (long long)p * n;
  uint8_t* out = passed + (long long)p * n;
  for (long long i = lo + threadIdx.x; i < hi; i += kSThreads) out[i] = row[i] >= sig ? 1 : 0;
}

__global__ void sig_output_kernel(int P, const SigState* __restrict__ st, double* __restrict__ sig_out,
                                  long long* __restrict__ nsig_out, int empty) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  sig_out[p] = empty ? key_value(kInfKey) : st[p].sig;
  nsig_out[p] = empty ? 0 : st[p].nsig;
}

inline size_t wal(size_t v) { return (v + 255) / 256 * 256; }

struct SigLayout {
  int nseg;
  long long cap;  // list capacity per particle (weights)
  size_t state, hist, rk, ri, rc, lk, li, lc, total;
};

SigLayout sig_layout(int P, long long n) {
  SigLayout L;
  L.nseg = (int)((n + kScanChunk - 1) / kScanChunk) * kWarps;
  L.cap = (long long)L.nseg * kSeg;
  const size_t pc = (size_t)P * (size_t)L.cap, ps = (size_t)P * (size_t)L.nseg;
  size_t o = 0;
  L.state = o;
  o += wal(sizeof(SigState) * P);
  L.hist = o;
  o += wal(sizeof(unsigned) * (size_t)P * kBuckets);
  L.rk = o;
  o += wal(sizeof(u64) * pc);
  L.ri = o;
  o += wal(sizeof(unsigned) * pc);
  L.rc = o;
  o += wal(sizeof(unsigned) * ps);
  L.lk = o;
  o += wal(sizeof(u64) * pc);
  L.li = o;
  o += wal(sizeof(unsigned) * pc);
  L.lc = o;
  o += wal(sizeof(unsigned) * ps);
  L.total = o;
  return L;
}

}  // namespace
}  // namespace b200d2

extern "C" size_t b200d2_significance_workspace(int P, long long n) {
  using namespace b200d2;
  if (P <= 0 || n <= 0) return 0;
  return sig_layout(P, n).total;
}

extern "C" int b200d2_significance(const double* d_weights, int P, long long n, const double* d_sum,
                                   double adaptive_fraction, long long max_significants, double* d_sig_weight,
                                   long long* d_nsig, uint8_t* d_passed, void* d_workspace, size_t workspace_bytes,
                                   void* stream) {
  using namespace b200d2;
  if (P < 0 || n < 0 || std::isnan(adaptive_fraction)) return B200D2_ERR_INVALID;
  if (P == 0) return B200D2_OK;
  if (!d_sig_weight || !d_nsig) return B200D2_ERR_INVALID;
  if (P > 65535 || n >= kMaxN) return B200D2_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    sig_output_kernel<<<(P + 127) / 128, 128, 0, s>>>(P, nullptr, d_sig_weight, d_nsig, 1);
    count_launch();
    return status_from_cuda(cudaGetLastError());
  }
  if (!d_weights || !d_sum) return B200D2_ERR_INVALID;
  const SigLayout W = sig_layout(P, n);
  if (!d_workspace || workspace_bytes < W.total) return B200D2_ERR_INVALID;
  uint8_t* ws = static_cast<uint8_t*>(d_workspace);
  SigState* st = reinterpret_cast<SigState*>(ws + W.state);
  unsigned* hist = reinterpret_cast<unsigned*>(ws + W.hist);
  u64* rk = reinterpret_cast<u64*>(ws + W.rk);
  unsigned* ri = reinterpret_cast<unsigned*>(ws + W.ri);
  unsigned* rc = reinterpret_cast<unsigned*>(ws + W.rc);
  u64* lk = reinterpret_cast<u64*>(ws + W.lk);
  unsigned* li = reinterpret_cast<unsigned*>(ws + W.li);
  unsigned* lc = reinterpret_cast<unsigned*>(ws + W.lc);
  // 16-byte loads of rows need even row lengths (row starts 16-byte aligned);
  // 8-byte mask stores need row lengths divisible by 8
  const int vec = (n % 2 == 0 && reinterpret_cast<uintptr_t>(d_weights) % 16 == 0) ? 1 : 0;
  const int vmask = (d_passed && n % 8 == 0 && reinterpret_cast<uintptr_t>(d_passed) % 8 == 0) ? 1 : 0;
  const u64* keys = reinterpret_cast<const u64*>(d_weights);

  // state (phase = sum, counters zero) and the histogram start at zero; every
  // reader of the histogram clears what it read
  B200D2_CUDA_TRY(cudaMemsetAsync(ws, 0, W.rk, s));
  const dim3 gscan((unsigned)((n + kScanChunk - 1) / kScanChunk), (unsigned)P);
  const dim3 glist(kLevelCtas, (unsigned)P);
  unsigned launches = 0;

  // sum phase: pass A, the binade range, pass B (with the first level's
  // counts), the first level, the deeper levels and the final step
  sig_scan_kernel<<<gscan, kSThreads, 0, s>>>(keys, n, vec, d_sum, adaptive_fraction, st, hist);
  sig_bracket_kernel<<<(P + 3) / 4, 128, 0, s>>>(st, P, hist, max_significants);
  sig_bin_kernel<<<gscan, kSThreads, 0, s>>>(keys, n, vec, vmask, W.cap, W.nseg, st, rk, ri, rc, hist, d_passed);
  sig_narrow_kernel<<<P, kSThreads, 0, s>>>(kPhaseSum, st, hist, max_significants);
  sig_level_kernel<<<glist, kSThreads, 0, s>>>(keys, rk, ri, rc, lk, li, lc, n, W.cap, W.nseg, kPhaseSum, st,
                                               d_passed);
  sig_deep_kernel<<<P, kSThreads, 0, s>>>(lk, li, lc, n, W.cap, W.nseg, kPhaseSum, st, max_significants, d_passed);
  launches += 6;
  if (max_significants > 0) {
    // rank phase (capped particles): the same levels by counts, from the array
    sig_count_kernel<<<gscan, kSThreads, 0, s>>>(keys, n, st, hist);
    sig_narrow_kernel<<<P, kSThreads, 0, s>>>(kPhaseRank, st, hist, max_significants);
    sig_level_kernel<<<glist, kSThreads, 0, s>>>(keys, rk, ri, rc, lk, li, lc, n, W.cap, W.nseg, kPhaseRank, st,
                                                 d_passed);
    sig_deep_kernel<<<P, kSThreads, 0, s>>>(lk, li, lc, n, W.cap, W.nseg, kPhaseRank, st, max_significants,
                                            d_passed);
    launches += 4;
  }
  if (d_passed) {
    sig_fullmask_kernel<<<gscan, kSThreads, 0, s>>>(d_weights, n, st, d_passed);
    ++launches;
  }
  sig_output_kernel<<<(P + 127) / 128, 128, 0, s>>>(P, st, d_sig_weight, d_nsig, 0);
  ++launches;
  count_launch(launches);
  return status_from_cuda(cudaGetLastError());
}
