// common.cuh -- device building blocks shared by every kernel of the sampler.
//
// Everything here is deterministic: integer arithmetic, or IEEE double
// operations written with explicit round-to-nearest intrinsics so that the
// compiler cannot contract them into FMAs.  The CPU oracle performs the same
// operations in the same order, so draws agree bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gpulda {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int32_t i32;
typedef int64_t i64;

constexpr u32 kFullMask = 0xffffffffu;

// Philox stream ids (counter word 3, low 8 bits).  The upper 24 bits of that
// word carry a sub-draw index for samplers that need more than one block of
// four words (Poisson rejection attempts).
enum Stream : u32 {
  kStreamInitCounts = 1,  // initial n from word counts (src/cu/polyaurn.cu:61-79)
  kStreamPhi = 2,         // x ~ Poisson(beta + n)   (src/cu/polyaurn.cu:87-123)
  kStreamZ = 3,           // topic draws              (src/cu/topics.cu:36-105)
  kStreamFoldInit = 4,    // fold-in: initial topics of a served document
  kStreamFold = 5,        // fold-in: topic draws of a served document
};

// Poisson inversion tables: rows n = 0..kPoisN-1 hold the CDF of
// Poisson(n + beta) as 32-bit thresholds, T[n][j] = min(floor(P(X<=j)*2^32),
// 2^32-1); the guide gives the first j with T[n][j] > b*2^24.
constexpr u32 kPoisN = 64;
constexpr u32 kPoisW = 192;
constexpr u32 kLogFacN = 256;
constexpr u32 kPtrsMaxAttempts = 64;

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Counter c[0..3], key k[0..1].
// ---------------------------------------------------------------------------
struct U4 {
  u32 x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, u32 k0, u32 k1) {
  constexpr u32 M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr u32 W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const u32 hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const u32 hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Counter layout: (index low, index high, iteration, stream | sub << 8).
__device__ __forceinline__ U4 draw4(u64 index, u32 t, u32 stream, u32 sub, u32 k0, u32 k1) {
  return philox4x32_10(U4{(u32)index, (u32)(index >> 32), t, stream | (sub << 8)}, k0, k1);
}

// 53-bit uniform double in [0, 1) from two words.
__device__ __forceinline__ double u53(u32 a, u32 b) {
  const u64 m = ((u64)(a >> 5) << 26) | (u64)(b >> 6);
  return __dmul_rn((double)m, 1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------
// Natural log from +, -, *, / only: x = m * 2^e with m in (sqrt(1/2), sqrt(2)],
// log m = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + ...), s = (m-1)/(m+1).
// |s| <= 0.1716, so 12 terms reach double precision.  Identical on host and
// device because every operation is correctly rounded.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double det_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -__longlong_as_double(0x7ff0000000000000LL)
                                   : __longlong_as_double(0x7ff8000000000000LL);
  u64 bits = (u64)__double_as_longlong(x);
  int e = (int)((bits >> 52) & 0x7ff) - 1023;
  double m = __longlong_as_double((long long)((bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
  if (m > 1.4142135623730951) {
    m = __dmul_rn(m, 0.5);
    e += 1;
  }
  const double s = __ddiv_rn(__dadd_rn(m, -1.0), __dadd_rn(m, 1.0));
  const double s2 = __dmul_rn(s, s);
  double p = 1.0 / 23.0;
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 21.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 19.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 17.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 15.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 13.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 11.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 9.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 7.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 5.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0 / 3.0);
  p = __dadd_rn(__dmul_rn(p, s2), 1.0);
  const double lm = __dmul_rn(__dmul_rn(2.0, s), p);
  return __dadd_rn(__dmul_rn((double)e, 0.6931471805599453), lm);
}

// log(k!) : table below kLogFacN, Stirling series above.
__device__ __forceinline__ double log_factorial(i64 k, const double* __restrict__ lfac) {
  if (k < (i64)kLogFacN) return lfac[k];
  const double x = (double)(k + 1);
  const double ix = __ddiv_rn(1.0, x);
  const double ix2 = __dmul_rn(ix, ix);
  // 1/(12x) - 1/(360x^3) + 1/(1260x^5)
  double corr = __dadd_rn(__dmul_rn(ix2, 1.0 / 1260.0), -1.0 / 360.0);
  corr = __dadd_rn(__dmul_rn(corr, ix2), 1.0 / 12.0);
  corr = __dmul_rn(corr, ix);
  double r = __dmul_rn(__dadd_rn(x, -0.5), det_log(x));
  r = __dadd_rn(r, -x);
  r = __dadd_rn(r, 0.91893853320467274);  // log(2 pi) / 2
  return __dadd_rn(r, corr);
}

struct PoisTables {
  const u32* cdf;     // kPoisN x kPoisW
  const uint8_t* guide;  // kPoisN x 256
  const double* lfac; // kLogFacN
};

// Poisson(lambda) for lambda >= 10 by transformed rejection with squeeze
// (W. Hoermann, "The transformed rejection method for generating Poisson
// random variables", Insurance: Mathematics and Economics 12, 1993).
// Attempt a uses Philox block (index, t, stream, 1 + a).
static __device__ __noinline__ u32 poisson_ptrs(double lam, u64 index, u32 t, u32 stream, u32 k0, u32 k1,
                                                const double* __restrict__ lfac) {
  const double slam = __dsqrt_rn(lam);
  const double loglam = det_log(lam);
  const double b = __dadd_rn(0.931, __dmul_rn(2.53, slam));
  const double a = __dadd_rn(-0.059, __dmul_rn(0.02483, b));
  const double inv_alpha = __dadd_rn(1.1239, __ddiv_rn(1.1328, __dadd_rn(b, -3.4)));
  const double vr = __dadd_rn(0.9277, -__ddiv_rn(3.6224, __dadd_rn(b, -2.0)));
  for (u32 att = 0; att < kPtrsMaxAttempts; ++att) {
    const U4 r = draw4(index, t, stream, 1 + att, k0, k1);
    const double U = __dadd_rn(u53(r.x, r.y), -0.5);
    const double V = u53(r.z, r.w);
    const double us = __dadd_rn(0.5, -fabs(U));
    const double kf = floor(__dadd_rn(__dadd_rn(__dmul_rn(__dadd_rn(__ddiv_rn(__dmul_rn(2.0, a), us), b), U), lam), 0.43));
    if (us >= 0.07 && V <= vr) return (u32)kf;
    if (kf < 0.0 || (us < 0.013 && V > us)) continue;
    const i64 k = (i64)kf;
    const double lhs = det_log(__ddiv_rn(__dmul_rn(V, inv_alpha), __dadd_rn(__ddiv_rn(a, __dmul_rn(us, us)), b)));
    const double rhs = __dadd_rn(__dadd_rn(-lam, __dmul_rn(kf, loglam)), -log_factorial(k, lfac));
    if (lhs <= rhs) return (u32)k;
  }
  return (u32)floor(lam);  // reached with probability far below 2^-100
}

// Cells share Philox blocks: cell c's inversion word is word (c & 3) of the
// block with counter index c >> 2 and sub-draw 0.
__device__ __forceinline__ u32 u4_word(const U4& r, u32 i) {
  return i == 0 ? r.x : i == 1 ? r.y : i == 2 ? r.z : r.w;
}

// x ~ Poisson(n + beta) for cell `index`.  n < kPoisN: inversion of the 32-bit
// CDF table with the cell's word `ru`; otherwise transformed rejection.
__device__ __forceinline__ u32 poisson_draw(u32 n, double beta, u32 ru, u64 index, u32 t, u32 stream,
                                            u32 k0, u32 k1, const PoisTables& tb) {
  if (n < kPoisN) {
    const u32* row = tb.cdf + (size_t)n * kPoisW;
    u32 j = tb.guide[n * 256u + (ru >> 24)];
    while (j < kPoisW - 1 && ru >= __ldg(row + j)) ++j;
    return j;
  }
  return poisson_ptrs(__dadd_rn((double)n, beta), index, t, stream, k0, k1, tb.lfac);
}

// Alias entry of a word's sparse table (one slot per topic with q > 0):
// bits 0-31 keep-threshold in units of 2^-32 of a slot, bits 32-47 the slot's
// own topic, bits 48-63 its alias topic.  The slot keeps its topic when r < threshold.
__device__ __forceinline__ u32 alias_pick(u64 entry, u32 r) {
  return r < (u32)entry ? (u32)(entry >> 32) & 0xffffu : (u32)(entry >> 48);
}

// floor(r * B / 2^32) for r < 2^32, exact.
__device__ __forceinline__ u64 scale_u32(u32 r, u64 B) {
  return (u64)r * (B >> 32) + (((u64)r * (B & 0xffffffffULL)) >> 32);
}

// Sparse-branch test: u * (alpha*A + B) < B with u = r / 2^32, in double.
__device__ __forceinline__ int take_sparse(u32 r, float alpha, u64 A, u64 B, int* degenerate) {
  const double tot = __dadd_rn(__dmul_rn((double)alpha, (double)A), (double)B);
  *degenerate = !(tot > 0.0);
  const double u = __dmul_rn((double)r, 1.0 / 4294967296.0);
  return __dmul_rn(u, tot) < (double)B;
}

// Threshold of an alias slot holding weight p (0 <= p <= A) out of capacity A.
__device__ __forceinline__ u32 alias_threshold(u64 p, u64 A) {
  if (A == 0 || p >= A) return 0xffffffffu;
  const double t = floor(__ddiv_rn(__dmul_rn((double)p, 4294967296.0), (double)A));
  return t >= 4294967295.0 ? 0xffffffffu : (u32)t;
}

}  // namespace gpulda
