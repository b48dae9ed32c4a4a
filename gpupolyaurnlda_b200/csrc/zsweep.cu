// zsweep.cu -- the per-document topic sweep (reference: sample_topics,
// src/cu/topics.cu:36-105, with count_topics / compute_product_cumsum /
// draw_wary_search / draw_alias from src/cu/topics.cuh:63-192).
//
// One warp per document; documents come from a global work counter.  The
// document's topic counts m_d live in shared memory as 16-bit counts plus a
// bitmap of nonzero topics.  Per token (after removing its current topic):
//   B      = sum_k m_dk * q[w][k]      (u64, exact)
//   sparse iff u0 * (alpha*A[w] + B) < B
//   sparse: target = floor(u1 * B); topic = first k in ascending order whose
//           inclusive prefix of m_dk * q[w][k] exceeds target
//   dense:  slot = floor(u2 * K); topic = slot if u3 < threshold else alias
//   (alpha*A + B == 0: the topic is kept)
// then the topic is added back and n[w][topic] incremented.
//
// B and the prefix run over the intersection of the document's topics and the
// word's nonzero q.  The warp walks whichever side is smaller: the document's
// bitmap (gathering q[w][k]) or the word's list of nonzero q (gathering m_dk
// from shared memory).  Either way each lane owns a contiguous range in
// ascending topic order, so lane order then position is ascending topic order
// and, the masses being exact integers, both walks select the same topic.
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
  u32 wpl;       // bitmap words per lane
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

__global__ void __launch_bounds__(256, 4) z_sweep_kernel(ZKernelArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32 K = m.K, V = m.V, wpl = a.wpl;
  const u32 Kp = (K + 63) & ~63u;
  const u32 nbw = 32 * wpl;
  const size_t per_warp = (size_t)Kp * 2 + (size_t)nbw * 4;
  uint16_t* cnt = (uint16_t*)(zsm + warp * per_warp);
  u32* bits = (u32*)(zsm + warp * per_warp + (size_t)Kp * 2);
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
    if (L > kMaxDocLen) {
      status |= kStatusDocTooLong;
      continue;
    }
    if (off + L > p.n_tokens) {
      status |= kStatusDocRange;
      continue;
    }
    for (u32 i = lane; i < Kp / 8; i += 32) reinterpret_cast<uint4*>(cnt)[i] = make_uint4(0, 0, 0, 0);
    for (u32 i = lane; i < nbw; i += 32) bits[i] = 0;
    __syncwarp();
    for (u32 i = lane; i < L; i += 32) {
      u32 k = p.z[off + i];
      if (k >= K) {
        status |= kStatusBadTopic;
        k %= K;
      }
      atomicAdd(reinterpret_cast<u32*>(cnt) + (k >> 1), 1u << ((k & 1) * 16));
      atomicOr(bits + (k >> 5), 1u << (k & 31));
    }
    __syncwarp();
    u32 nz = 0;  // distinct topics in the document (warp-uniform)
    for (u32 b = 0; b < wpl; ++b) nz += __popc(bits[lane * wpl + b]);
    nz = (u32)warp_sum_u64(nz);

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
      // Per-token word data for the whole chunk, loaded lane-parallel so the
      // token loop never waits on them: nnz, dense mass, and the alias entry
      // of the slot this token's dense draw would use.
      const u32 my_s = (u32)(((u64)r.z * K) >> 32);
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u64 my_al = valid ? __ldg(m.al + (size_t)my_w * K + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      for (u32 j = 0; j < nt; ++j) {
        const u32 wj = __shfl_sync(kFullMask, my_w, j);
        const u32 zj = __shfl_sync(kFullMask, my_z, j);
        const u32 r0 = __shfl_sync(kFullMask, r.x, j);
        const u32 r1 = __shfl_sync(kFullMask, r.y, j);
        const size_t row = (size_t)wj * K;
        const u32* __restrict__ qrow = m.q + row;
        const u64* __restrict__ crow = m.csr + row;
        const u32 nw = __shfl_sync(kFullMask, my_nw, j);
        const u64 Aw = __shfl_sync(kFullMask, my_A, j);
        if (j + 1 < nt) {
          // Warm L1 with the next token's lines: this lane's q line and the
          // start of its share of the word's nonzero list.
          const u32 wn = __shfl_sync(kFullMask, my_w, j + 1);
          const u32 nn = __shfl_sync(kFullMask, my_nw, j + 1);
          const size_t rn = (size_t)wn * K;
          if (lane * wpl * 32 < K) asm volatile("prefetch.global.L1 [%0];" ::"l"(m.q + rn + lane * wpl * 32));
          const u32 cn = (nn + 31) >> 5;
          if (lane * cn < nn) asm volatile("prefetch.global.L1 [%0];" ::"l"(m.csr + rn + lane * cn));
        }
        u32 emptied = 0;
        if (lane == 0) {
          const u32 c = cnt[zj] - 1u;
          cnt[zj] = (uint16_t)c;
          if (c == 0) {
            bits[zj >> 5] &= ~(1u << (zj & 31));
            emptied = 1;
          }
        }
        nz -= __shfl_sync(kFullMask, emptied, 0);
        __syncwarp();
        // Sparse mass over this lane's contiguous range.
        const bool word_side = nw < nz;
        const u32 cper = (nw + 31) >> 5;
        u64 ls = 0;
        if (word_side) {
          const u32 e0 = min(nw, lane * cper), e1 = min(nw, e0 + cper);
          for (u32 e = e0; e < e1; ++e) {
            const u64 ent = __ldg(crow + e);
            ls += (u64)cnt[(u32)ent & 0xffffu] * (u32)(ent >> 32);
          }
        } else {
          for (u32 b = 0; b < wpl; ++b) {
            const u32 wi = lane * wpl + b;
            u32 bm = bits[wi];
            while (bm) {
              const u32 k = wi * 32 + (__ffs(bm) - 1);
              bm &= bm - 1;
              ls += (u64)cnt[k] * __ldg(qrow + k);
            }
          }
        }
        const u64 incl = warp_incl_scan_u64(ls, lane);
        const u64 B = __shfl_sync(kFullMask, incl, 31);
        int degenerate;
        const int sp = take_sparse(r0, m.alpha, Aw, B, &degenerate);
        u32 k = zj;
        if (!degenerate) {
          if (sp) {
            const u64 target = scale_u32(r1, B);
            const u32 f = __ffs(__ballot_sync(kFullMask, incl > target)) - 1;
            u64 run = __shfl_sync(kFullMask, incl - ls, f);
            // Finish inside lane f's range, 32 candidates at a time.
            if (word_side) {
              const u32 e0 = min(nw, f * cper), e1 = min(nw, e0 + cper);
              for (u32 s0 = e0; s0 < e1; s0 += 32) {
                const u32 e = s0 + lane;
                u64 mass = 0;
                u32 kk = 0;
                if (e < e1) {
                  const u64 ent = __ldg(crow + e);
                  kk = (u32)ent & 0xffffu;
                  mass = (u64)cnt[kk] * (u32)(ent >> 32);
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
              for (u32 b = 0; b < wpl; ++b) {
                const u32 wi = f * wpl + b;
                const u32 bm = bits[wi];
                const u32 kk = wi * 32 + lane;
                u64 mass = 0;
                if ((bm >> lane) & 1u) mass = (u64)cnt[kk] * __ldg(qrow + kk);
                const u64 in2 = warp_incl_scan_u64(mass, lane);
                const u64 tot = __shfl_sync(kFullMask, in2, 31);
                if (run + tot > target) {
                  const u32 jj = __ffs(__ballot_sync(kFullMask, run + in2 > target)) - 1;
                  k = wi * 32 + jj;
                  break;
                }
                run += tot;
              }
            }
          } else {
            const u32 r3 = __shfl_sync(kFullMask, r.w, j);
            const u32 s = __shfl_sync(kFullMask, my_s, j);
            const u64 e = __shfl_sync(kFullMask, my_al, j);
            k = alias_pick(e, s, r3);
          }
        }
        u32 filled = 0;
        if (lane == 0) {
          const u32 c = cnt[k] + 1u;
          cnt[k] = (uint16_t)c;
          if (c == 1) {
            bits[k >> 5] |= 1u << (k & 31);
            filled = 1;
          }
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
        nz += __shfl_sync(kFullMask, filled, 0);
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (valid) p.z[off + i] = new_z;
    }
    if (lane == 0 && p.K_d) p.K_d[doc] = nz;
    if (want_ll) {
      double dl = 0.0;
      for (u32 b = 0; b < wpl; ++b) {
        const u32 wi = lane * wpl + b;
        u32 bm = bits[wi];
        while (bm) {
          const u32 k = wi * 32 + (__ffs(bm) - 1);
          bm &= bm - 1;
          dl += lgamma((double)m.alpha + (double)cnt[k]) - a.lg_a;
        }
      }
      dl = warp_sum_f64(dl);
      if (lane == 0) ll_acc += dl + a.lg_Ka - lgamma((double)K * (double)m.alpha + (double)L);
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
    if (want_ll) {
      atomicAdd(p.ll, ll_acc);
      atomicAdd(p.ll + 1, ll_skip);
    }
  }
  status = __reduce_or_sync(kFullMask, status);
  if (lane == 0 && status) atomicOr(p.status, status);
}

}  // namespace

size_t z_sweep_smem_per_warp(u32 K) {
  const u32 Kp = (K + 63) & ~63u;
  const u32 nw = (K + 31) / 32;
  const u32 wpl = (nw + 31) / 32;
  return (size_t)Kp * 2 + (size_t)32 * wpl * 4;
}

void launch_z_sweep(const ModelDev& m, const ZLaunch& z, cudaStream_t s) {
  if (!z.n_docs) return;
  ZKernelArgs a;
  a.m = m;
  a.z = z;
  const u32 nw = (m.K + 31) / 32;
  a.wpl = (nw + 31) / 32;
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  const size_t per_warp = z_sweep_smem_per_warp(m.K);
  // Warps per block: as many as fit the shared-memory budget, at most 8.
  u32 wpb = 8;
  while (wpb > 1 && per_warp * wpb > kZMaxSmem) --wpb;
  const size_t smem = per_warp * wpb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(z_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, z_sweep_kernel, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (z.n_docs + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  z_sweep_kernel<<<blocks, 32 * wpb, smem, s>>>(a);
}

}  // namespace gpulda
