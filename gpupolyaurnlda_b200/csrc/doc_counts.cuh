// doc_counts.cuh -- one document's topic counts in shared memory and the
// per-token topic draw, shared by the Gibbs sweep (zsweep.cu) and the
// fold-in of new documents against a fixed model (serve.cu).
//
// Reference: sample_topics / count_topics / compute_product_cumsum /
// draw_wary_search / draw_alias, src/cu/topics.cu:36-105 and
// src/cu/topics.cuh:63-192.  One warp owns one document.  Its counts m_d are
// a dense array of 16-bit counts plus the sorted list of its nonzero topics.
// Per token (after removing its current topic):
//   B      = sum_k m_dk * q[w][k]      (u64, exact)
//   sparse iff u0 * (alpha*A[w] + B) < B
//   sparse: target = floor(u1 * B); topic = first k in ascending order whose
//           inclusive prefix of m_dk * q[w][k] exceeds target
//   dense:  slot = floor(u2 * nnz[w]) of the word's alias table; topic = the
//           slot's own topic if u3 < threshold, else its alias
//   (alpha*A + B == 0: the topic is kept)
// then the topic is added back.
//
// B and the prefix run over the intersection of the document's topics and the
// word's nonzero q.  The warp walks whichever list is shorter: the document's
// sorted topic list (gathering q[w][k]) or the word's list of nonzero q
// (gathering m_dk from shared memory).  Either way lane l takes the l-th
// contiguous chunk of an ascending list, so lane order then position is
// ascending topic order and, the masses being exact integers, both walks
// select the same topic.
#pragma once

#include "common.cuh"
#include "warp.cuh"

namespace gpulda {

// Dead list entries (topics whose count fell to zero) tolerated before the
// list is compacted.  Each costs every walk of the document's list one
// zero-mass element; a compaction costs a pass over the list.  Measured on the
// mid corpus (K=1000), fifth iteration: 0 -> 37.2 ms per sweep, 4 -> 36.6,
// 8 -> 36.8, 16 -> 37.2, 32 -> 38.2, 64 -> 39.3.
constexpr u32 kMaxDead = 4;

// Shared memory per warp for documents of up to Kmax topics: the 16-bit
// counts (Kmax rounded up to 32 entries: the list build scans them 32 at a
// time) and the sorted list (at most Kmax distinct topics, rounded up to 8
// entries).  Both parts are multiples of 16 bytes.  Every byte counts here:
// shared memory comes out of the SM's 256 KB L1, and the q gathers of the
// walk live on L1 hits (mid corpus: 1.6 KB more per warp took the carveout
// from 196 to 228 KB, L1 from 60 to 28 KB, and the sweep from 2.72e9 to
// 2.30e9 tokens/s).
__host__ __device__ __forceinline__ size_t doc_counts_bytes(u32 Kmax) {
  return (size_t)((Kmax + 31) & ~31u) * 2 + (size_t)((Kmax + 7) & ~7u) * 2;
}

struct DocCounts {
  uint16_t* cnt;  // dense counts, Kmax rounded up to 32 entries
  // Sorted topics of the document: every topic with a nonzero count, plus
  // topics whose count fell to zero since the last compaction (their mass is
  // zero, so they never change B or the selected topic).  Entries are
  // distinct topics, so the list never holds more than K.
  uint16_t* tl;
  u32 nz;    // topics with a nonzero count
  u32 nl;    // list length (nz plus dead entries)
};

__device__ __forceinline__ DocCounts doc_counts_at(unsigned char* base, u32 Kmax) {
  DocCounts dc;
  dc.cnt = (uint16_t*)base;
  dc.tl = dc.cnt + ((Kmax + 31) & ~31u);
  dc.nz = dc.nl = 0;
  return dc;
}

// First index i in the sorted list tl[0..n) with tl[i] >= k (warp-cooperative).
__device__ __forceinline__ u32 list_lower_bound(const uint16_t* tl, u32 n, u32 k, u32 lane) {
  u32 lo = 0;
  while (n > 32) {
    const u32 step = (n + 31) >> 5;
    const u32 idx = lo + lane * step;
    const bool lt = lane * step < n && tl[idx] < k;
    u32 c = __popc(__ballot_sync(kFullMask, lt));
    if (c == 0) c = 1;
    lo += (c - 1) * step;
    n = min(step, n - (c - 1) * step);
  }
  const bool lt = lane < n && tl[lo + lane] < k;
  return lo + __popc(__ballot_sync(kFullMask, lt));
}

// Drops the entries of topics whose count is zero from the list tl[0..n)
// (stable, in place, warp-cooperative).  Returns the new length.
__device__ __forceinline__ u32 list_compact(uint16_t* tl, u32 n, const uint16_t* cnt, u32 lane) {
  u32 out = 0;
  for (u32 b = 0; b < n; b += 32) {
    const u32 e = b + lane;
    const u32 k = e < n ? tl[e] : 0u;
    const bool keep = e < n && cnt[k] != 0;
    const u32 ball = __ballot_sync(kFullMask, keep);
    __syncwarp();
    if (keep) tl[out + __popc(ball & ((1u << lane) - 1u))] = (uint16_t)k;
    out += __popc(ball);
    __syncwarp();
  }
  return out;
}

// Inserts k at tl[pos] in a list of n entries (warp-cooperative shift right).
__device__ __forceinline__ void list_insert(uint16_t* tl, u32 n, u32 pos, u32 k, u32 lane) {
  for (u32 top = n; top > pos; top = top > pos + 32 ? top - 32 : pos) {
    const u32 src = top - 1 - lane;
    const bool act = lane < top - pos && lane < 32;
    const uint16_t v = act ? tl[src] : 0;
    __syncwarp();
    if (act) tl[src + 1] = v;
    __syncwarp();
  }
  if (lane == 0) tl[pos] = (uint16_t)k;
  __syncwarp();
}

// Counts and sorted list of the topics z[0..L) of a document with K topics.
// A topic >= K is counted modulo K and reported in *status.
__device__ __forceinline__ void doc_counts_build(DocCounts& dc, const u32* z, u32 L, u32 K, u32 lane, u32* status,
                                                 u32 bad_topic_bit) {
  const u32 Kp = (K + 31) & ~31u;
  for (u32 i = lane; i < Kp / 8; i += 32) reinterpret_cast<uint4*>(dc.cnt)[i] = make_uint4(0, 0, 0, 0);
  __syncwarp();
  for (u32 i = lane; i < L; i += 32) {
    u32 k = z[i];
    if (k >= K) {
      *status |= bad_topic_bit;
      k %= K;
    }
    atomicAdd(reinterpret_cast<u32*>(dc.cnt) + (k >> 1), 1u << ((k & 1) * 16));
  }
  __syncwarp();
  // Sorted list, 32 topics per round: lane l tests topic b + l (consecutive
  // 16-bit loads, free of bank conflicts, where a contiguous range per lane
  // would put the lanes' loads 64 bytes apart); the round's ballot gives each
  // nonzero topic its list position.
  const u32 below = (1u << lane) - 1u;
  u32 pos = 0;
  for (u32 b = 0; b < Kp; b += 32) {
    const bool nz = dc.cnt[b + lane] != 0;
    const u32 m = __ballot_sync(kFullMask, nz);
    if (nz) dc.tl[pos + __popc(m & below)] = (uint16_t)(b + lane);
    pos += __popc(m);
  }
  __syncwarp();
  dc.nz = dc.nl = pos;
}

// One token (lane j's in the current chunk): removes topic zj, draws the new
// topic, adds it back.  r0/r1 are the token's uniform words (already
// broadcast); my_r3 / my_al are lane j's fourth word and the alias entry of
// its dense slot (broadcast only when the dense branch runs).  qrow / crow are
// the word's fixed-point Phi row and nonzero list, nw its list length, Aw its
// dense mass.  Returns the topic; *nz_minus receives the document's distinct
// topics without the token, *sparse whether the sparse branch chose it.
// kRegChunk: the longest per-lane chunk kept in registers (lists up to 32 x
// kRegChunk entries need no second pass); 6 for the single-model sweep (mid
// corpus: 4 -> 36.8 ms, 6 -> 36.3, 8 -> 42.1 with spills), 4 where the caller
// holds more registers of its own (the batched sweep and the fold-in spill at
// 6; the 64-problem batched workload ran at 2.43e9 tokens/s with 6 against
// 2.64e9 with 4).
template <u32 kRegChunk = 6>
__device__ __forceinline__ u32 token_step(DocCounts& dc, u32 zj, u32 r0, u32 r1, u32 my_r3, u64 my_al, u32 j,
                                          const u32* __restrict__ qrow, const u64* __restrict__ crow, u32 nw, u64 Aw,
                                          float alpha, u32 lane, u32* nz_minus, bool* sparse) {
  uint16_t* cnt = dc.cnt;
  uint16_t* tl = dc.tl;
  // remove the token's current topic
  const u32 cz = cnt[zj];
  __syncwarp();
  if (lane == 0) cnt[zj] = (uint16_t)(cz - 1u);
  if (cz == 1u) --dc.nz;  // the entry stays in the list until compaction
  __syncwarp();
  const u32 nl = dc.nl;
  // the shorter list (mid corpus: taking the word's list up to 0.8x, 1.5x or 2x
  // the document's gave 2.71e9, 2.72e9 and 2.68e9 tokens/s against 2.77e9)
  const bool word_side = nw < nl;
  // Sparse mass over this lane's contiguous chunk.
  const u32 len = word_side ? nw : nl;
  const u32 cper = (len + 31) >> 5;
  const u32 e0 = min(len, lane * cper), e1 = min(len, e0 + cper);
  // Chunks of at most kRegChunk elements (lists up to 32 kRegChunk entries): unrolled
  // independent loads, masses kept in registers, so the selection needs no
  // second pass; the crossing element's topic is read once afterwards.
  const bool in_regs = cper <= kRegChunk;
  u64 ms[kRegChunk];
  u64 ls = 0;
  if (in_regs) {
    const u32 n_my = e1 - e0;
    if (word_side) {
      u64 ent[kRegChunk];
#pragma unroll
      for (u32 c = 0; c < kRegChunk; ++c) ent[c] = c < n_my ? __ldg(crow + e0 + c) : 0ull;
#pragma unroll
      for (u32 c = 0; c < kRegChunk; ++c) ms[c] = (u64)cnt[(u32)ent[c] & 0xffffu] * (u32)(ent[c] >> 32);
    } else {
      u32 ks[kRegChunk], qs[kRegChunk];
#pragma unroll
      for (u32 c = 0; c < kRegChunk; ++c) ks[c] = c < n_my ? (u32)tl[e0 + c] : 0u;
#pragma unroll
      for (u32 c = 0; c < kRegChunk; ++c) qs[c] = c < n_my ? __ldg(qrow + ks[c]) : 0u;
#pragma unroll
      for (u32 c = 0; c < kRegChunk; ++c) ms[c] = (u64)cnt[ks[c]] * qs[c];
    }
#pragma unroll
    for (u32 c = 0; c < kRegChunk; ++c) ls += ms[c];
  } else if (word_side) {
    for (u32 e = e0; e < e1; ++e) {
      const u64 ent = __ldg(crow + e);
      ls += (u64)cnt[(u32)ent & 0xffffu] * (u32)(ent >> 32);
    }
  } else {
    for (u32 e = e0; e < e1; ++e) {
      const u32 k = tl[e];
      ls += (u64)cnt[k] * __ldg(qrow + k);
    }
  }
  const u64 incl = warp_incl_scan_u64(ls, lane);
  const u64 B = __shfl_sync(kFullMask, incl, 31);
  int degenerate;
  const int sp = take_sparse(r0, alpha, Aw, B, &degenerate);
  u32 k = zj;
  if (!degenerate) {
    if (sp) {
      const u64 target = scale_u32(r1, B);
      const u32 f = __ffs(__ballot_sync(kFullMask, incl > target)) - 1;
      if (in_regs) {
        // Lane f's first element whose inclusive prefix exceeds the target
        // (prefixes grow with c, so going down the last hit is the first);
        // every lane computes its own, lane f's is broadcast.
        u64 pre = incl - ls;
        u32 cx = kRegChunk - 1;
#pragma unroll
        for (u32 c = kRegChunk - 1; c-- > 0;) {
          u64 t = pre;
#pragma unroll
          for (u32 d = 0; d <= c; ++d) t += ms[d];
          if (t > target) cx = c;
        }
        const u32 ef = f * cper + __shfl_sync(kFullMask, cx, f);
        k = word_side ? ((u32)__ldg(crow + ef) & 0xffffu) : (u32)tl[ef];
      } else {
        u64 run = __shfl_sync(kFullMask, incl - ls, f);
        // Finish inside lane f's chunk, 32 candidates at a time.
        const u32 f0 = min(len, f * cper), f1 = min(len, f0 + cper);
        for (u32 s0 = f0; s0 < f1; s0 += 32) {
          const u32 e = s0 + lane;
          u64 mass = 0;
          u32 kk = 0;
          if (e < f1) {
            if (word_side) {
              const u64 ent = __ldg(crow + e);
              kk = (u32)ent & 0xffffu;
              mass = (u64)cnt[kk] * (u32)(ent >> 32);
            } else {
              kk = tl[e];
              mass = (u64)cnt[kk] * __ldg(qrow + kk);
            }
          }
          const u64 in2 = warp_incl_scan_u64(mass, lane);
          const u64 tot = __shfl_sync(kFullMask, in2, 31);
          if (run + tot > target) {
            const u32 jj = __ffs(__ballot_sync(kFullMask, run + in2 > target)) - 1;
            k = __shfl_sync(kFullMask, kk, jj);
            break;
          }
          run += tot;
        }
      }
    } else {
      const u32 r3 = __shfl_sync(kFullMask, my_r3, j);
      const u64 e = __shfl_sync(kFullMask, my_al, j);
      k = alias_pick(e, r3);
    }
  }
  *sparse = sp && !degenerate;
  *nz_minus = dc.nz;
  // add the new topic
  const u32 ck = cnt[k];
  __syncwarp();
  if (lane == 0) cnt[k] = (uint16_t)(ck + 1u);
  if (ck == 0u) {
    ++dc.nz;
    // A topic back from zero may still be in the list as a dead entry; the
    // search that finds the insert position tells.
    const u32 pos = list_lower_bound(tl, dc.nl, k, lane);
    if (pos == dc.nl || tl[pos] != k) {
      list_insert(tl, dc.nl, pos, k, lane);
      ++dc.nl;
    }
  }
  if (dc.nl - dc.nz > kMaxDead) dc.nl = list_compact(tl, dc.nl, cnt, lane);
  return k;
}

// sum over the document's topics of lgamma(alpha + m_dk) - lgamma(alpha)
// (warp-reduced, every lane receives it).
__device__ __forceinline__ double doc_lgamma_sum(const DocCounts& dc, float alpha, double lg_a, u32 lane) {
  double dl = 0.0;
  for (u32 e = lane; e < dc.nl; e += 32) {
    const u32 c = dc.cnt[dc.tl[e]];
    if (c) dl += lgamma((double)alpha + (double)c) - lg_a;
  }
  return warp_sum_f64(dl);
}

}  // namespace gpulda
