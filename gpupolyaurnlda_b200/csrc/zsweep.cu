// zsweep.cu -- the per-document topic sweep (reference: sample_topics,
// src/cu/topics.cu:36-105, with count_topics / compute_product_cumsum /
// draw_wary_search / draw_alias from src/cu/topics.cuh:63-192).
//
// One warp per document; documents come from a global work counter (longest
// first when an order is given).  The document's counts and the per-token
// draw are in doc_counts.cuh; this kernel adds the count rebuild
// n[w][k] += 1 for every token's new topic, the statistics and the joint
// log-likelihood.
#include <algorithm>
#include <cmath>

#include "doc_counts.cuh"
#include "kernels.cuh"

namespace gpulda {

namespace {

constexpr u32 kMaxDocLen = 65535u;
constexpr size_t kZMaxSmem = 200 * 1024;
constexpr size_t kTokStageBytes = 32 * 32;  // per warp: 32 tokens x 32 bytes

struct ZKernelArgs {
  ModelDev m;
  ZLaunch z;
  BatchDev b;    // problem tables (batched launches only)
  u32 Kmax;      // largest K of the launch (sets the shared-memory stride)
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

// BATCH: the launch sweeps documents of many independent problems laid out in
// one set of arenas; each document's K, alpha, Philox key and token numbering
// come from its problem, and a token's (word, topic) row starts at
// b.row_off[w] instead of w * K.  Otherwise all parameters come from `m`.
//
// LL: the launch accumulates the joint log-likelihood.  A separate
// instantiation, so the sweep without it keeps no log-likelihood registers
// live: the kernel runs at 64 registers per thread (four 256-thread blocks
// per SM), where every live register is felt.  For the same reason the
// statistics live in shared memory (per-chunk sums of at most 22 bits in one
// register), not in per-thread 64-bit counters.
template <bool BATCH, bool LL>
__global__ void __launch_bounds__(256, 4) z_sweep_kernel(ZKernelArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  __shared__ unsigned long long blk_stats[4];  // tokens, documents, sparse work, sparse draws
  if (threadIdx.x < 4) blk_stats[threadIdx.x] = 0;
  __syncthreads();
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32 V = m.V;
  unsigned char* wsm = zsm + (size_t)warp * (doc_counts_bytes(a.Kmax) + kTokStageBytes);
  DocCounts dc = doc_counts_at(wsm, a.Kmax);
  uint4* stage = reinterpret_cast<uint4*>(wsm + doc_counts_bytes(a.Kmax));
  const bool want_ll = LL;

  // log-likelihood terms, accumulated per lane
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
    u32 K = m.K, key0 = m.key0, key1 = m.key1, pb = 0;
    float alpha = m.alpha;
    u64 tok_base = p.tok_base;
    double lg_a = a.lg_a, lg_Ka = a.lg_Ka;
    const u32* __restrict__ t_ptr = p.t_dev;
    if (BATCH) {
      pb = a.b.pid[doc];
      K = a.b.K[pb];
      alpha = a.b.alpha[pb];
      key0 = a.b.key0[pb];
      key1 = a.b.key1[pb];
      tok_base = a.b.tok_base[pb];  // the problem's first token: local numbering
      lg_a = a.b.lg_a[pb];
      lg_Ka = a.b.lg_Ka[pb];
    }
    const u32 t = t_ptr ? *t_ptr : p.t;
    if (L > kMaxDocLen) {
      status |= kStatusDocTooLong;
      continue;
    }
    if (off + L > p.n_tokens) {
      status |= kStatusDocRange;
      continue;
    }
    doc_counts_build(dc, p.z + off, L, K, lane, &status, kStatusBadTopic);

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
      // Philox index: the token's position in its corpus (batched problems
      // count from their own first token) plus the buffer's offset.
      const U4 r = draw4(BATCH ? off + i - tok_base : tok_base + off + i, t, kStreamZ, 0, key0, key1);
      // Per-token word data for the whole chunk, loaded lane-parallel so the
      // token loop never waits on them: nnz, dense mass, and the alias entry
      // of the slot this token's dense draw would use.
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
      const u64 my_row = BATCH ? (valid ? __ldg(a.b.row_off + my_w) : 0ull) : (u64)my_w * K;
      const u64 my_al = (valid && my_nw) ? __ldg(m.al + my_row + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      // sum over the chunk of (min(nz without the token, nnz[w]) << 6) + sparse
      // (the first term at most 32 * 2048, the second at most 32)
      u32 chunk_st = 0;
      // The chunk's per-token data is staged in shared memory and read back
      // with two 16-byte broadcast loads per token instead of eight
      // shuffles: shuffles and shared loads share the L1 data pipe, which
      // bounds this kernel.
      __syncwarp();
      stage[2 * lane] = make_uint4(my_z, r.x, r.y, my_nw);
      stage[2 * lane + 1] = make_uint4((u32)my_row, (u32)(my_row >> 32), (u32)my_A, (u32)(my_A >> 32));
      __syncwarp();
      for (u32 j = 0; j < nt; ++j) {
        const uint4 s0 = stage[2 * j], s1 = stage[2 * j + 1];
        const u32 zj = s0.x, r0 = s0.y, r1 = s0.z, nw = s0.w;
        const size_t row = ((u64)s1.y << 32) | s1.x;
        const u64 Aw = ((u64)s1.w << 32) | s1.z;
        u32 nzm;
        bool sp;
        // The walk's elements per lane are known before the token's removal
        // (the list keeps dead entries), so the register path runs with as
        // few unrolled slots as the chunk needs: 2, 4 or 6 for the single
        // model (mid corpus, eighth iteration: 34.1 ms per sweep against
        // 36.4 ms with 6 slots for every token; one instantiation per
        // possible length spilled and took 67 ms), 2 or 4 for a batched launch
        // (64-problem batch: 2.83e9 tokens/s against 2.61e9).
        const u32 cper_j = ((nw < dc.nl ? nw : dc.nl) + 31) >> 5;
        u32 k;
#define TOKEN_STEP(R) \
  token_step<R>(dc, zj, r0, r1, r.w, my_al, j, m.q + row, m.csr + row, nw, Aw, alpha, lane, &nzm, &sp)
        if (cper_j <= 2)
          k = TOKEN_STEP(2u);
        else if (BATCH || cper_j <= 4)
          k = TOKEN_STEP(4u);
        else
          k = TOKEN_STEP(6u);
#undef TOKEN_STEP
        if (lane == 0) {
          atomicAdd(m.n + row + k, 1u);
          chunk_st += (min(nzm, nw) << 6) + (sp ? 1u : 0u);
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
    if (lane == 0 && p.K_d) p.K_d[doc] = dc.nz;
    if (want_ll) {
      const double dl = doc_lgamma_sum(dc, alpha, lg_a, lane);
      if (lane == 0) ll_acc += dl + lg_Ka - lgamma((double)K * (double)alpha + (double)L);
      if (BATCH) {  // per-problem sums
        const double s0 = warp_sum_f64(ll_acc), s1 = warp_sum_f64(ll_skip);
        if (lane == 0) {
          atomicAdd(p.ll + 2 * pb, s0);
          atomicAdd(p.ll + 2 * pb + 1, s1);
        }
        ll_acc = ll_skip = 0.0;
      }
    }
    if (lane == 0) {
      atomicAdd(blk_stats + 0, (unsigned long long)L);
      atomicAdd(blk_stats + 1, 1ull);
    }
    __syncwarp();
  }
  if (want_ll && !BATCH) {
    ll_acc = warp_sum_f64(ll_acc);
    ll_skip = warp_sum_f64(ll_skip);
  }
  if (lane == 0 && want_ll && !BATCH) {
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

template <bool BATCH, bool LL>
void launch_impl(const ZKernelArgs& a, u32 n_docs, cudaStream_t s, u32 wpb, u32 blocks_per_sm) {
  const size_t per_warp = doc_counts_bytes(a.Kmax) + kTokStageBytes;
  // Warps per block: as many as fit the shared-memory budget (at most the request).
  while (wpb > 1 && per_warp * wpb > kZMaxSmem) --wpb;
  const size_t smem = per_warp * wpb;
  // The ceiling, not this launch's size: captured graphs may hold launches of
  // several sizes.
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(z_sweep_kernel<BATCH, LL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kZMaxSmem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, z_sweep_kernel<BATCH, LL>, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  if (blocks_per_sm && (int)blocks_per_sm < per_sm) per_sm = (int)blocks_per_sm;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (n_docs + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  z_sweep_kernel<BATCH, LL><<<blocks, 32 * wpb, smem, s>>>(a);
}

}  // namespace

void launch_z_sweep(const ModelDev& m, const ZLaunch& z, cudaStream_t s) {
  if (!z.n_docs) return;
  ZKernelArgs a;
  a.m = m;
  a.z = z;
  a.b = BatchDev{};
  a.Kmax = m.K;
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  if ((z.flags & 1u) && z.ll)
    launch_impl<false, true>(a, z.n_docs, s, 8, 0);
  else
    launch_impl<false, false>(a, z.n_docs, s, 8, 0);
}

void launch_z_sweep_batch(const ModelDev& arenas, const BatchDev& b, u32 Kmax, const ZLaunch& z, cudaStream_t s,
                          u32 warps_per_block, u32 blocks_per_sm) {
  if (!z.n_docs) return;
  ZKernelArgs a;
  a.m = arenas;
  a.z = z;
  a.b = b;
  a.Kmax = Kmax;
  a.lg_a = 0;
  a.lg_Ka = 0;
  if ((z.flags & 1u) && z.ll)
    launch_impl<true, true>(a, z.n_docs, s, warps_per_block, blocks_per_sm);
  else
    launch_impl<true, false>(a, z.n_docs, s, warps_per_block, blocks_per_sm);
}

}  // namespace gpulda
