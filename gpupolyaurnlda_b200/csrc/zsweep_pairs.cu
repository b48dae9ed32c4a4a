// zsweep_pairs.cu -- the z sweep for large K with each document's topic counts
// as a sorted list of (topic, count) pairs in shared memory (reference: the
// per-document HashMap of src/cu/hashmap.cuh:13-334 used by sample_topics,
// src/cu/topics.cu:36-105).
//
// The list is the order-preserving map of zsweep_map.cu without empty slots:
// entries (topic << 16 | count), ascending topic.  A topic whose count falls
// to zero stays as a dead entry (zero mass, so it never changes B or the
// selected topic) and is revived if the topic returns; more than kPairsMaxDead
// dead entries are compacted away.  Lookups are warp-cooperative 32-ary searches
// (two ballot rounds for lists up to 1024 entries); inserts shift the tail.
// The walk reads the entries in ascending topic order, so the sparse draw is
// identical to the dense-count kernel's, the map kernel's and the CPU
// oracle's.
//
// Per token the warp walks (i) the document's entries, gathering q[w][k]
// (counts come with the entries), or (ii) the word's list of nonzero q, each
// lane finding its topics' counts by binary search in the document's entries,
// whichever is cheaper (below).  Lane l takes the l-th contiguous chunk of the walked
// list; chunks of at most 4 elements keep their masses in registers, so the
// sparse selection needs no second pass.
//
// Capacity per warp: min(lmax, K) live entries, at most kPairsMaxDead + 1
// dead ones before a compaction, rounded up: min(lmax, K) + 64.  An insert that would pass it is
// refused and reported (it cannot happen under that bound).
#include <algorithm>
#include <cmath>

#include "kernels.cuh"
#include "warp.cuh"

namespace {
// Dead entries tolerated before a compaction: each costs every walk of the
// document's entries one zero-mass element, a compaction one pass.  At
// K=10000 (D = 2e6) 8 gave 129 ms per sweep against 133 ms for 16 and 141 ms
// for 32.
constexpr unsigned kPairsMaxDead = 8;
}  // namespace

namespace gpulda {

namespace {

constexpr u32 kMaxDocLen = 65535u;
constexpr size_t kTokStageBytes = 32 * 32;  // per warp: 32 tokens x 32 bytes
constexpr u32 kStatusListFull = 32;         // an insert found the list full (cannot happen)

struct PairArgs {
  ModelDev m;
  ZLaunch z;
  u32 cap;       // entries per warp
  u32 lmax;      // longest document this launch accepts
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

__device__ __forceinline__ u32 topic_of(u32 e) { return e >> 16; }
__device__ __forceinline__ u32 count_of(u32 e) { return e & 0xffffu; }

// First index i in P[0..n) with topic(P[i]) >= k (warp-cooperative).
__device__ __forceinline__ u32 pairs_lower_bound(const u32* P, u32 n, u32 k, u32 lane) {
  u32 lo = 0;
  while (n > 32) {
    const u32 step = (n + 31) >> 5;
    const bool lt = lane * step < n && topic_of(P[lo + lane * step]) < k;
    u32 c = __popc(__ballot_sync(kFullMask, lt));
    if (c == 0) c = 1;
    lo += (c - 1) * step;
    n = min(step, n - (c - 1) * step);
  }
  const bool lt = lane < n && topic_of(P[lo + lane]) < k;
  return lo + __popc(__ballot_sync(kFullMask, lt));
}

// First index i in P[0..n) with topic(P[i]) >= k, by one lane's binary search.
__device__ __forceinline__ u32 pairs_find(const u32* P, u32 n, u32 k) {
  u32 lo = 0, hi = n;
  while (lo < hi) {
    const u32 mid = (lo + hi) >> 1;
    if (topic_of(P[mid]) < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Count of topic k in P[0..n) by one lane's binary search.
__device__ __forceinline__ u32 pairs_count(const u32* P, u32 n, u32 k) {
  u32 lo = 0, hi = n;
  while (lo < hi) {
    const u32 mid = (lo + hi) >> 1;
    if (topic_of(P[mid]) < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && topic_of(P[lo]) == k) ? count_of(P[lo]) : 0u;
}

// Inserts e at P[pos] in a list of n entries (warp-cooperative shift right).
__device__ __forceinline__ void pairs_insert(u32* P, u32 n, u32 pos, u32 e, u32 lane) {
  for (u32 top = n; top > pos; top = top > pos + 32 ? top - 32 : pos) {
    const u32 src = top - 1 - lane;
    const bool act = lane < top - pos;
    const u32 v = act ? P[src] : 0u;
    __syncwarp();
    if (act) P[src + 1] = v;
    __syncwarp();
  }
  if (lane == 0) P[pos] = e;
  __syncwarp();
}

// Drops dead entries (stable, in place); returns the new length.
__device__ __forceinline__ u32 pairs_compact(u32* P, u32 n, u32 lane) {
  u32 out = 0;
  for (u32 b = 0; b < n; b += 32) {
    const u32 i = b + lane;
    const u32 e = i < n ? P[i] : 0u;
    const bool keep = i < n && count_of(e) != 0;
    const u32 ball = __ballot_sync(kFullMask, keep);
    __syncwarp();
    if (keep) P[out + __popc(ball & ((1u << lane) - 1u))] = e;
    out += __popc(ball);
    __syncwarp();
  }
  return out;
}

// Count of topic k += 1 at its position; inserts it if absent.  bm (may be
// null): the bitmap of topics with a positive count, kept in step.
__device__ __forceinline__ void pairs_add_at(u32* P, u32& nl, u32& nz, u32 pos, u32 k, u32 cap, u32 lane,
                                             u32* status, u32* bm) {
  const u32 e = pos < nl ? P[pos] : 0xffffffffu;
  __syncwarp();
  if (pos < nl && topic_of(e) == k) {
    if (lane == 0) {
      P[pos] = e + 1u;
      if (bm && count_of(e) == 0) bm[k >> 5] |= 1u << (k & 31);
    }
    if (count_of(e) == 0) ++nz;  // a dead entry revived
    __syncwarp();
    return;
  }
  if (nl >= cap) {
    *status |= kStatusListFull;
    return;
  }
  pairs_insert(P, nl, pos, (k << 16) | 1u, lane);
  if (bm && lane == 0) bm[k >> 5] |= 1u << (k & 31);
  __syncwarp();
  ++nl;
  ++nz;
}

// Launches whose documents are at most this long keep the topic bitmap.
constexpr u32 kBitmapMaxLen = 1024;

// Whether topic k has a positive count (always true without the bitmap: the
// caller then searches).
template <bool BM>
__device__ __forceinline__ bool in_doc(const u32* bm, u32 k) {
  return !BM || ((bm[k >> 5] >> (k & 31)) & 1u);
}

// One token's draw over the document's entries P[0..nl) (bm: the optional
// topic bitmap) and the word's row: the walk of the shorter side split into
// 32 contiguous chunks, chunks of at most R elements kept in registers.
// Returns the topic; *pos_out receives its entry when the document-side walk
// found it (else 0xffffffff).
template <bool BM, u32 R>
__device__ __forceinline__ u32 pairs_draw(const u32* P, u32 nl, const u32* bm, const u32* __restrict__ qrow,
                                          const u64* __restrict__ crow, u32 nw, u64 Aw, float alpha, bool word_side,
                                          u32 zj, u32 r0, u32 r1, u32 my_r3, u64 my_al, u32 j, u32 lane,
                                          u32* pos_out, int* sp_out, int* degenerate_out) {
  const u32 len = word_side ? nw : nl;
  const u32 cper = (len + 31) >> 5;
  const u32 e0 = min(len, lane * cper), e1 = min(len, e0 + cper);
  const bool in_regs = cper <= R;
  u64 ms[R];
  u64 ls = 0;
  if (in_regs) {
    const u32 n_my = e1 - e0;
    if (word_side) {
#pragma unroll
      for (u32 c = 0; c < R; ++c) {
        const u64 ent = c < n_my ? __ldg(crow + e0 + c) : 0ull;
        ms[c] = c < n_my && in_doc<BM>(bm, (u32)ent & 0xffffu)
                    ? (u64)pairs_count(P, nl, (u32)ent & 0xffffu) * (u32)(ent >> 32)
                    : 0ull;
      }
    } else {
      u32 es[R], qs[R];
#pragma unroll
      for (u32 c = 0; c < R; ++c) es[c] = c < n_my ? P[e0 + c] : 0u;
#pragma unroll
      for (u32 c = 0; c < R; ++c) qs[c] = c < n_my ? __ldg(qrow + topic_of(es[c])) : 0u;
#pragma unroll
      for (u32 c = 0; c < R; ++c) ms[c] = (u64)count_of(es[c]) * qs[c];
    }
#pragma unroll
    for (u32 c = 0; c < R; ++c) ls += ms[c];
  } else if (word_side) {
    for (u32 e = e0; e < e1; ++e) {
      const u64 ent = __ldg(crow + e);
      if (in_doc<BM>(bm, (u32)ent & 0xffffu))
        ls += (u64)pairs_count(P, nl, (u32)ent & 0xffffu) * (u32)(ent >> 32);
    }
  } else {
    for (u32 e = e0; e < e1; ++e) {
      const u32 en = P[e];
      ls += (u64)count_of(en) * __ldg(qrow + topic_of(en));
    }
  }
  const u64 incl = warp_incl_scan_u64(ls, lane);
  const u64 B = __shfl_sync(kFullMask, incl, 31);
  int degenerate;
  const int sp = take_sparse(r0, alpha, Aw, B, &degenerate);
  *sp_out = sp;
  *degenerate_out = degenerate;
  u32 k = zj;
  u32 pos = 0xffffffffu;  // the new topic's entry, when the walk found it
  if (!degenerate) {
    if (sp) {
      const u64 target = scale_u32(r1, B);
      const u32 f = __ffs(__ballot_sync(kFullMask, incl > target)) - 1;
      u32 ef;
      if (in_regs) {
        // lane f's first element whose inclusive prefix exceeds the target
        u64 pre = incl - ls;
        u32 cx = R - 1;
#pragma unroll
        for (u32 c = R - 1; c-- > 0;) {
          u64 t = pre;
#pragma unroll
          for (u32 d = 0; d <= c; ++d) t += ms[d];
          if (t > target) cx = c;
        }
        ef = f * cper + __shfl_sync(kFullMask, cx, f);
      } else {
        u64 run = __shfl_sync(kFullMask, incl - ls, f);
        const u32 f0 = min(len, f * cper), f1 = min(len, f0 + cper);
        ef = f1 - 1;
        for (u32 s0 = f0; s0 < f1; s0 += 32) {
          const u32 e = s0 + lane;
          u64 mass = 0;
          if (e < f1) {
            if (word_side) {
              const u64 ent = __ldg(crow + e);
              if (in_doc<BM>(bm, (u32)ent & 0xffffu))
                mass = (u64)pairs_count(P, nl, (u32)ent & 0xffffu) * (u32)(ent >> 32);
            } else {
              const u32 en = P[e];
              mass = (u64)count_of(en) * __ldg(qrow + topic_of(en));
            }
          }
          const u64 in2 = warp_incl_scan_u64(mass, lane);
          const u64 tot = __shfl_sync(kFullMask, in2, 31);
          if (run + tot > target) {
            ef = s0 + __ffs(__ballot_sync(kFullMask, run + in2 > target)) - 1;
            break;
          }
          run += tot;
        }
      }
      if (word_side) {
        k = (u32)__ldg(crow + ef) & 0xffffu;
      } else {
        k = topic_of(P[ef]);
        pos = ef;
      }
    } else {
      const u32 r3 = __shfl_sync(kFullMask, my_r3, j);
      const u64 e = __shfl_sync(kFullMask, my_al, j);
      k = alias_pick(e, r3);
    }
  }
  *pos_out = pos;
  return k;
}

// Shared memory per warp: entries, staged token data, and the bitmap.
__host__ __device__ __forceinline__ size_t pairs_warp_bytes(u32 cap, u32 K, bool bm) {
  return (size_t)cap * 4 + kTokStageBytes + (bm ? ((((size_t)K + 31) / 32 * 4 + 15) & ~(size_t)15) : 0);
}

// Four blocks per SM (64 registers, no spills).  LL: the launch accumulates
// the joint log-likelihood (a separate instantiation, so the plain sweep keeps
// no log-likelihood registers); the statistics are per-chunk sums in one
// register, flushed to per-block shared counters.  At K=10000 the whole
// sweep (long-document launch, then short-document launch) takes 446 ms over
// 8e6 documents and 109 ms over 2e6, against 483 and 131 ms at three blocks.
//
// BM (launches whose lists are short, lmax <= kBitmapMaxLen): each warp also
// keeps a bitmap of the topics with a positive count.  The document's entries
// are then built from it (bitmap of the tokens' topics, its set bits in order,
// then one binary search and shared-memory atomic per token) instead of one
// warp-cooperative insert per token, and a word-side walk skips the binary
// search of every word topic absent from the document (most of them; a lane
// slot where no lane's topic is present costs no search at all).
template <bool LL, bool BM>
__global__ void __launch_bounds__(256, 4) z_sweep_pairs_kernel(PairArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  __shared__ unsigned long long blk_stats[4];  // tokens, documents, sparse work, sparse draws
  if (threadIdx.x < 4) blk_stats[threadIdx.x] = 0;
  __syncthreads();
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32 K = m.K, V = m.V;
  const u32 bmw = (K + 31) >> 5;  // bitmap words
  unsigned char* wsm = zsm + (size_t)warp * pairs_warp_bytes(a.cap, K, BM);
  u32* P = (u32*)wsm;
  uint4* stage = (uint4*)(wsm + (size_t)a.cap * 4);
  u32* bm = BM ? (u32*)(wsm + (size_t)a.cap * 4 + kTokStageBytes) : nullptr;
  const bool want_ll = LL;

  double ll_acc = 0.0, ll_skip = 0.0;
  u32 status = 0;

  while (true) {
    u32 doc = 0;
    if (lane == 0) doc = atomicAdd(p.work, 1u);
    doc = __shfl_sync(kFullMask, doc, 0);
    if (doc >= p.n_docs) break;
    if (p.order) doc = p.order[doc];
    const u32 L = p.d_len[doc];
    const u64 off = p.d_idx[doc];
    if (L > kMaxDocLen || L > a.lmax) {
      status |= kStatusDocTooLong;
      continue;
    }
    if (off + L > p.n_tokens) {
      status |= kStatusDocRange;
      continue;
    }
    // build the sorted entries of the document's topics
    u32 nl = 0, nz = 0;
    if (BM) {
      for (u32 i = lane; i < bmw; i += 32) bm[i] = 0;
      __syncwarp();
      for (u32 i = lane; i < L; i += 32) {
        u32 k = p.z[off + i];
        if (k >= K) {
          status |= kStatusBadTopic;
          k %= K;
        }
        atomicOr(bm + (k >> 5), 1u << (k & 31));
      }
      __syncwarp();
      // the set bits in ascending order, 32 words per round
      for (u32 b = 0; b < bmw; b += 32) {
        const u32 wi = b + lane;
        u32 bits = wi < bmw ? bm[wi] : 0u;
        const u32 c = __popc(bits);
        u32 x = c;
#pragma unroll
        for (u32 o = 1; o < 32; o <<= 1) {
          const u32 y = __shfl_up_sync(kFullMask, x, o);
          if (lane >= o) x += y;
        }
        u32 pos = nl + x - c;
        while (bits) {
          P[pos++] = (wi * 32 + (u32)(__ffs(bits) - 1)) << 16;
          bits &= bits - 1;
        }
        nl += __shfl_sync(kFullMask, x, 31);
      }
      __syncwarp();
      // counts: one binary search and shared-memory atomic per token
      for (u32 i = lane; i < L; i += 32) {
        const u32 k = p.z[off + i] % K;
        atomicAdd(P + pairs_find(P, nl, k), 1u);
      }
      __syncwarp();
      nz = nl;
    } else {
      for (u32 i = 0; i < L; ++i) {
        u32 k = p.z[off + i];
        if (k >= K) {
          status |= kStatusBadTopic;
          k %= K;
        }
        pairs_add_at(P, nl, nz, pairs_lower_bound(P, nl, k, lane), k, a.cap, lane, &status, nullptr);
      }
    }

    for (u32 base = 0; base < L; base += 32) {
      const u32 i = base + lane;
      const bool valid = i < L;
      u32 my_w = valid ? p.w[off + i] : 0;
      u32 my_z = valid ? p.z[off + i] : 0;
      if (my_w >= V) {
        status |= kStatusBadWord;
        my_w %= V;
      }
      if (my_z >= K) my_z %= K;
      const U4 r = draw4(p.tok_base + off + i, p.t, kStreamZ, 0, m.key0, m.key1);
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
      const u64 my_row = (u64)my_w * K;
      const u64 my_al = (valid && my_nw) ? __ldg(m.al + my_row + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      // sum over the chunk of (min(nz without the token, nnz[w]) << 6) + sparse
      // (the first term at most 32 * 32768, the second at most 32)
      u32 chunk_st = 0;
      __syncwarp();
      stage[2 * lane] = make_uint4(my_z, r.x, r.y, my_nw);
      stage[2 * lane + 1] = make_uint4((u32)my_row, (u32)(my_row >> 32), (u32)my_A, (u32)(my_A >> 32));
      __syncwarp();
      for (u32 j = 0; j < nt; ++j) {
        const uint4 s0 = stage[2 * j], s1 = stage[2 * j + 1];
        const u32 zj = s0.x, r0 = s0.y, r1 = s0.z, nw = s0.w;
        const size_t row = ((u64)s1.y << 32) | s1.x;
        const u64 Aw = ((u64)s1.w << 32) | s1.z;
        const u32* __restrict__ qrow = m.q + row;
        const u64* __restrict__ crow = m.csr + row;
        // remove the token's current topic (present with a positive count)
        {
          const u32 pz = pairs_lower_bound(P, nl, zj, lane);
          const u32 e = pz < nl ? P[pz] : 0u;
          __syncwarp();
          if (pz < nl && topic_of(e) == zj && count_of(e) > 0) {
            if (lane == 0) {
              P[pz] = e - 1u;
              if (BM && count_of(e) == 1) bm[zj >> 5] &= ~(1u << (zj & 31));
            }
            if (count_of(e) == 1) --nz;
          }
          __syncwarp();
        }
        // The word's list is read contiguously while the document side
        // gathers scattered q values from rows of 4 K bytes (mostly beyond L2 at
        // large K), so the word side is taken up to 4x the document's length
        // (measured best at K=10000 among 1x, 2x, 4x, 8x; again with the
        // topic bitmap, on 2e6 documents: 103 ms per sweep against 116 for
        // 2x, 115 for 8x and 126 for 16x).
        const bool word_side = nw < 4 * nl;
        // as few register slots as the walk's chunks need: 2, 4 or 6 (K=10000,
        // 2e6 documents: 101.8 ms per sweep against 102.9 with 2 or 4; an 8-slot
        // path beside them spilled and took 108.4)
        const u32 cper_j = ((word_side ? nw : nl) + 31) >> 5;
        u32 pos;
        int sp, degenerate;
        u32 k = cper_j <= 2 ? pairs_draw<BM, 2>(P, nl, bm, qrow, crow, nw, Aw, m.alpha, word_side, zj, r0, r1, r.w, my_al,
                                                 j, lane, &pos, &sp, &degenerate)
                : cper_j <= 4 ? pairs_draw<BM, 4>(P, nl, bm, qrow, crow, nw, Aw, m.alpha, word_side, zj, r0, r1, r.w, my_al,
                                                 j, lane, &pos, &sp, &degenerate)
                            : pairs_draw<BM, 6>(P, nl, bm, qrow, crow, nw, Aw, m.alpha, word_side, zj, r0, r1, r.w, my_al,
                                                 j, lane, &pos, &sp, &degenerate);
        const u32 nzm = nz;
        if (pos == 0xffffffffu) pos = pairs_lower_bound(P, nl, k, lane);
        pairs_add_at(P, nl, nz, pos, k, a.cap, lane, &status, bm);
        if (nl - nz > kPairsMaxDead) nl = pairs_compact(P, nl, lane);
        if (lane == 0) {
          atomicAdd(m.n + row + k, 1u);
          chunk_st += (min(nzm, nw) << 6) + ((sp && !degenerate) ? 1u : 0u);
        }
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (lane == 0) {
        atomicAdd(blk_stats + 2, (unsigned long long)(chunk_st >> 6));
        atomicAdd(blk_stats + 3, (unsigned long long)(chunk_st & 63u));
      }
      if (valid) {
        p.z[off + i] = new_z;
        if (want_ll) {  // log Phi[new topic][word], one token per lane
          const u32 qk = __ldg(m.q + my_row + new_z);
          if (qk)
            ll_acc += log((double)qk) - 22.18070977791825;  // 32 log 2
          else
            ll_skip += 1.0;
        }
      }
    }
    if (lane == 0 && p.K_d) p.K_d[doc] = nz;
    if (want_ll) {
      double dl = 0.0;
      for (u32 e = lane; e < nl; e += 32) {
        const u32 c = count_of(P[e]);
        if (c) dl += lgamma((double)m.alpha + (double)c) - a.lg_a;
      }
      dl = warp_sum_f64(dl);
      if (lane == 0) ll_acc += dl + a.lg_Ka - lgamma((double)K * (double)m.alpha + (double)L);
    }
    if (lane == 0) {
      atomicAdd(blk_stats + 0, (unsigned long long)L);
      atomicAdd(blk_stats + 1, 1ull);
    }
    __syncwarp();
  }
  if (want_ll) {
    ll_acc = warp_sum_f64(ll_acc);
    ll_skip = warp_sum_f64(ll_skip);
  }
  if (lane == 0 && want_ll) {
    atomicAdd(p.ll, ll_acc);
    atomicAdd(p.ll + 1, ll_skip);
  }
  status = __reduce_or_sync(kFullMask, status);
  if (lane == 0 && status) atomicOr(p.status, status);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(p.counters + kCtrTokens, blk_stats[0]);
    atomicAdd(p.counters + kCtrDocs, blk_stats[1]);
    atomicAdd(p.counters + kCtrSparseWork, blk_stats[2]);
    atomicAdd(p.counters + kCtrSparseDraws, blk_stats[3]);
  }
}

}  // namespace

u32 z_pairs_cap(u32 K, u32 lmax) { return ((std::min(std::max(lmax, 1u), K) + 64 + 31) / 32) * 32; }

bool launch_z_sweep_pairs(const ModelDev& m, const ZLaunch& z, cudaStream_t s, u32 lmax) {
  if (!z.n_docs) return true;
  PairArgs a;
  a.m = m;
  a.z = z;
  a.lmax = lmax;
  a.cap = z_pairs_cap(m.K, lmax);
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  const bool bmap = lmax <= kBitmapMaxLen;
  const size_t per_warp = pairs_warp_bytes(a.cap, m.K, bmap);
  constexpr size_t kBudget = 200 * 1024;
  u32 wpb = 8;
  while (wpb > 1 && per_warp * wpb > kBudget) --wpb;
  if (per_warp * wpb > kBudget) return false;
  const size_t smem = per_warp * wpb;
  const bool ll = (z.flags & 1u) && z.ll;
  auto kern = bmap ? (ll ? z_sweep_pairs_kernel<true, true> : z_sweep_pairs_kernel<false, true>)
                   : (ll ? z_sweep_pairs_kernel<true, false> : z_sweep_pairs_kernel<false, false>);
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBudget);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (z.n_docs + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  kern<<<blocks, 32 * wpb, smem, s>>>(a);
  return true;
}

}  // namespace gpulda
