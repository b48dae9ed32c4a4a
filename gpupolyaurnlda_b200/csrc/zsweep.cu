// zsweep.cu -- the per-document topic sweep (reference: sample_topics,
// src/cu/topics.cu:36-105, with count_topics / compute_product_cumsum /
// draw_wary_search / draw_alias from src/cu/topics.cuh:63-192).
//
// One warp per document; documents come from a global work counter (longest
// first when an order is given).  The document's topic counts m_d live in
// shared memory as a dense array of 16-bit counts plus the sorted list of its
// nonzero topics.  Per token (after removing its current topic):
//   B      = sum_k m_dk * q[w][k]      (u64, exact)
//   sparse iff u0 * (alpha*A[w] + B) < B
//   sparse: target = floor(u1 * B); topic = first k in ascending order whose
//           inclusive prefix of m_dk * q[w][k] exceeds target
//   dense:  slot = floor(u2 * K); topic = slot if u3 < threshold else alias
//   (alpha*A + B == 0: the topic is kept)
// then the topic is added back and n[w][topic] incremented.
//
// B and the prefix run over the intersection of the document's topics and the
// word's nonzero q.  The warp walks whichever list is shorter: the document's
// sorted topic list (gathering q[w][k]) or the word's list of nonzero q
// (gathering m_dk from shared memory).  Either way lane l takes the l-th
// contiguous chunk of an ascending list, so lane order then position is
// ascending topic order and, the masses being exact integers, both walks
// select the same topic.
#include <algorithm>
#include <cmath>

#include "kernels.cuh"
#include "warp.cuh"

namespace gpulda {

namespace {

constexpr u32 kMaxDocLen = 65535u;
constexpr size_t kZMaxSmem = 200 * 1024;

struct ZKernelArgs {
  ModelDev m;
  ZLaunch z;
  BatchDev b;    // problem tables (batched launches only)
  u32 Kmax;      // largest K of the launch (sets the shared-memory stride)
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};


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
// (stable, in place, warp-cooperative) and clears their in-list bits.
// Returns the new length.
__device__ __forceinline__ u32 list_compact(uint16_t* tl, u32 n, const uint16_t* cnt, u32* inl, u32 lane) {
  u32 out = 0;
  for (u32 b = 0; b < n; b += 32) {
    const u32 e = b + lane;
    const u32 k = e < n ? tl[e] : 0u;
    const bool keep = e < n && cnt[k] != 0;
    const u32 ball = __ballot_sync(kFullMask, keep);
    __syncwarp();
    if (keep) tl[out + __popc(ball & ((1u << lane) - 1u))] = (uint16_t)k;
    if (e < n && !keep) atomicAnd(inl + (k >> 5), ~(1u << (k & 31)));
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

// Shared memory per warp: counts and list (2 x Kp u16) and the in-list bitmap.
__host__ __device__ __forceinline__ size_t z_warp_bytes(u32 K) {
  const size_t Kp = (K + 63) & ~63u;
  return Kp * 4 + ((Kp / 8 + 15) & ~(size_t)15);
}

// BATCH: the launch sweeps documents of many independent problems laid out in
// one set of arenas; each document's K, alpha, Philox key and token numbering
// come from its problem, and a token's (word, topic) row starts at
// b.row_off[w] instead of w * K.  Otherwise all parameters come from `m`.
template <bool BATCH>
__global__ void __launch_bounds__(256, 4) z_sweep_kernel(ZKernelArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32 V = m.V;
  const u32 Kpmax = (a.Kmax + 63) & ~63u;
  uint16_t* cnt = (uint16_t*)(zsm + (size_t)warp * z_warp_bytes(a.Kmax));
  // Sorted topics of the document: every topic with a nonzero count, plus
  // topics whose count fell to zero since the last compaction (their mass is
  // zero, so they never change B or the selected topic).
  uint16_t* tl = cnt + Kpmax;
  u32* inl = (u32*)(tl + Kpmax);  // bitmap: topic is in tl
  const bool want_ll = (p.flags & 1u) && p.ll;

  u64 st_tok = 0, st_docs = 0, st_S = 0, st_sp = 0;
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
    const u32 Kp = (K + 63) & ~63u;
    if (L > kMaxDocLen) {
      status |= kStatusDocTooLong;
      continue;
    }
    if (off + L > p.n_tokens) {
      status |= kStatusDocRange;
      continue;
    }
    for (u32 i = lane; i < Kp / 8; i += 32) reinterpret_cast<uint4*>(cnt)[i] = make_uint4(0, 0, 0, 0);
    for (u32 i = lane; i < Kp / 32; i += 32) inl[i] = 0;
    __syncwarp();
    for (u32 i = lane; i < L; i += 32) {
      u32 k = p.z[off + i];
      if (k >= K) {
        status |= kStatusBadTopic;
        k %= K;
      }
      atomicAdd(reinterpret_cast<u32*>(cnt) + (k >> 1), 1u << ((k & 1) * 16));
    }
    __syncwarp();
    // Sorted list of the nonzero topics: lane l compacts its contiguous range.
    u32 nz;
    {
      const u32 per = Kp / 32;
      const u32 k0 = lane * per;
      u32 c = 0;
      for (u32 k = k0; k < k0 + per; ++k) c += cnt[k] != 0;
      u32 pos = c;
#pragma unroll
      for (u32 o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(kFullMask, pos, o);
        if (lane >= o) pos += y;
      }
      nz = __shfl_sync(kFullMask, pos, 31);
      pos -= c;
      for (u32 k = k0; k < k0 + per; ++k)
        if (cnt[k]) {
          tl[pos++] = (uint16_t)k;
          atomicOr(inl + (k >> 5), 1u << (k & 31));
        }
      __syncwarp();
    }
    u32 nl = nz;  // list length (nz plus dead entries)

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
      // the dense draw's slot in the word's sparse alias table (nnz slots)
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
      const u64 my_row = BATCH ? (valid ? __ldg(a.b.row_off + my_w) : 0ull) : (u64)my_w * K;
      const u64 my_al = (valid && my_nw) ? __ldg(m.al + my_row + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      for (u32 j = 0; j < nt; ++j) {
        const u32 wj = __shfl_sync(kFullMask, my_w, j);
        const u32 zj = __shfl_sync(kFullMask, my_z, j);
        const u32 r0 = __shfl_sync(kFullMask, r.x, j);
        const u32 r1 = __shfl_sync(kFullMask, r.y, j);
        const size_t row = BATCH ? (size_t)__shfl_sync(kFullMask, my_row, j) : (size_t)wj * K;
        const u32* __restrict__ qrow = m.q + row;
        const u64* __restrict__ crow = m.csr + row;
        const u32 nw = __shfl_sync(kFullMask, my_nw, j);
        const u64 Aw = __shfl_sync(kFullMask, my_A, j);
        // remove the token's current topic
        const u32 cz = cnt[zj];
        __syncwarp();
        if (lane == 0) cnt[zj] = (uint16_t)(cz - 1u);
        if (cz == 1u) --nz;  // the entry stays in the list until compaction
        __syncwarp();
        const bool word_side = nw < nl;
        // Sparse mass over this lane's contiguous chunk.
        const u32 len = word_side ? nw : nl;
        const u32 cper = (len + 31) >> 5;
        const u32 e0 = min(len, lane * cper), e1 = min(len, e0 + cper);
        u64 ls = 0;
        if (word_side) {
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
          } else {
            const u32 r3 = __shfl_sync(kFullMask, r.w, j);
            const u64 e = __shfl_sync(kFullMask, my_al, j);
            k = alias_pick(e, r3);
          }
        }
        // add the new topic
        const u32 ck = cnt[k];
        __syncwarp();
        if (lane == 0) {
          cnt[k] = (uint16_t)(ck + 1u);
          atomicAdd(m.n + row + k, 1u);
          st_S += min(nz, nw);
          st_sp += (sp && !degenerate) ? 1 : 0;
          if (want_ll) {
            const u32 qk = __ldg(qrow + k);
            if (qk)
              ll_acc += log((double)qk) - 22.18070977791825;  // 32 log 2
            else
              ll_skip += 1.0;
          }
        }
        if (ck == 0u) {
          ++nz;
          if (!((inl[k >> 5] >> (k & 31)) & 1u)) {
            list_insert(tl, nl, list_lower_bound(tl, nl, k, lane), k, lane);
            if (lane == 0) atomicOr(inl + (k >> 5), 1u << (k & 31));
            __syncwarp();
            ++nl;
          }
        }
        if (nl - nz > 32u) nl = list_compact(tl, nl, cnt, inl, lane);
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (valid) p.z[off + i] = new_z;
    }
    if (lane == 0 && p.K_d) p.K_d[doc] = nz;
    if (want_ll) {
      double dl = 0.0;
      for (u32 e = lane; e < nl; e += 32) {
        const u32 c = cnt[tl[e]];
        if (c) dl += lgamma((double)alpha + (double)c) - lg_a;
      }
      dl = warp_sum_f64(dl);
      if (lane == 0) ll_acc += dl + lg_Ka - lgamma((double)K * (double)alpha + (double)L);
      if (BATCH) {  // per-problem sums
        if (lane == 0) {
          atomicAdd(p.ll + 2 * pb, ll_acc);
          atomicAdd(p.ll + 2 * pb + 1, ll_skip);
        }
        ll_acc = ll_skip = 0.0;
      }
    }
    st_tok += L;
    st_docs += 1;
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(p.counters + kCtrTokens, (unsigned long long)st_tok);
    atomicAdd(p.counters + kCtrDocs, (unsigned long long)st_docs);
    atomicAdd(p.counters + kCtrSparseWork, (unsigned long long)st_S);
    atomicAdd(p.counters + kCtrSparseDraws, (unsigned long long)st_sp);
    if (want_ll && !BATCH) {
      atomicAdd(p.ll, ll_acc);
      atomicAdd(p.ll + 1, ll_skip);
    }
  }
  status = __reduce_or_sync(kFullMask, status);
  if (lane == 0 && status) atomicOr(p.status, status);
}

template <bool BATCH>
void launch_impl(const ZKernelArgs& a, u32 n_docs, cudaStream_t s, u32 wpb, u32 blocks_per_sm) {
  const size_t per_warp = z_warp_bytes(a.Kmax);
  // Warps per block: as many as fit the shared-memory budget (at most the request).
  while (wpb > 1 && per_warp * wpb > kZMaxSmem) --wpb;
  const size_t smem = per_warp * wpb;
  // The ceiling, not this launch's size: captured graphs may hold launches of
  // several sizes.
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(z_sweep_kernel<BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kZMaxSmem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, z_sweep_kernel<BATCH>, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  if (blocks_per_sm && (int)blocks_per_sm < per_sm) per_sm = (int)blocks_per_sm;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (n_docs + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  z_sweep_kernel<BATCH><<<blocks, 32 * wpb, smem, s>>>(a);
}

}  // namespace

size_t z_sweep_smem_per_warp(u32 K) { return z_warp_bytes(K); }

void launch_z_sweep(const ModelDev& m, const ZLaunch& z, cudaStream_t s) {
  if (!z.n_docs) return;
  ZKernelArgs a;
  a.m = m;
  a.z = z;
  a.b = BatchDev{};
  a.Kmax = m.K;
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  launch_impl<false>(a, z.n_docs, s, 8, 0);
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
  launch_impl<true>(a, z.n_docs, s, warps_per_block, blocks_per_sm);
}

}  // namespace gpulda
