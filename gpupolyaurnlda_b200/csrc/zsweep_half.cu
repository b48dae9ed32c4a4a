// zsweep_half.cu -- the per-document topic sweep with two documents per warp
// (reference: sample_topics, src/cu/topics.cu:36-105, with count_topics /
// compute_product_cumsum / draw_wary_search / draw_alias from
// src/cu/topics.cuh:63-192), for models of at most 1024 topics.
//
// Each half-warp (16 lanes) owns one document and fetches its next document
// from the launch's work counter on its own; the two halves of a warp sweep
// their documents' tokens in lockstep, so every per-token step that does not
// scale with the document's topic list -- reading the staged token data,
// removing and adding the token's topic, the mixture test, the dense draw,
// the count rebuild -- is one warp instruction for two tokens.  The sparse
// walk over the shorter of the document's topic list and the word's nonzero
// list is split into 16 contiguous chunks per document (lane order, then
// position, is ascending topic order), reduced with a 16-lane u64 scan, and
// the crossing element is found in the owning lane's registers.  The draw is
// the one of doc_counts.cuh's token_step, so the result equals the
// one-warp-per-document kernel's and the oracle's bit for bit.
//
// Control flow stays warp-uniform around every warp-collective operation:
// per-half differences (document lengths, walk side, chunk sizes, inserts,
// compactions) are predicated, and loops whose trip counts differ between the
// halves run to the larger count with the other half idle.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "warp.cuh"

namespace gpulda {

namespace {

constexpr u32 kHalfMaxK = 1024;                 // topics per model of this kernel
constexpr u32 kHalfMaxDocLen = 65535u;          // 16-bit counts
constexpr u32 kHalfDead = 4;                    // dead list entries tolerated before compaction
constexpr u32 kHalfRegs = 8;                    // chunk elements kept in registers (lists <= 128)
constexpr u32 kHalfBatch = 4;                   // further chunk elements loaded per unrolled batch
constexpr u32 kHalfWarps = 12;                  // warps per block (24 documents)
// The word's nonzero list is walked while it is shorter than this many times
// the document's topic list: its entries are read contiguously (few cache
// lines per element), where the document side gathers q from across the row.
constexpr u32 kWordSideFactor = 1;
constexpr size_t kHalfSlotBytes = kHalfMaxK * 2 /* counts */ + kHalfMaxK * 2 /* list */ +
                                  kHalfMaxK / 8 /* in-list bitmap */ + 16 * 32 /* staged tokens */;
static_assert(kHalfSlotBytes % 128 == 0, "slot size");
// Slots are 64 bytes further apart than they need: the two halves of a warp
// then sit 16 banks apart, so their same-index reads (staged token data,
// broadcast counts) do not conflict.
constexpr size_t kHalfSlotStride = kHalfSlotBytes + 64;

struct HalfArgs {
  ModelDev m;
  ZLaunch z;
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

__device__ __forceinline__ u32 half_ballot(bool p, u32 hb) { return (__ballot_sync(kFullMask, p) >> hb) & 0xffffu; }

__device__ __forceinline__ u64 half_incl_scan_u64(u64 x, u32 hl) {
#pragma unroll
  for (u32 o = 1; o < 16; o <<= 1) {
    const u64 y = __shfl_up_sync(kFullMask, x, o, 16);
    if (hl >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ double half_sum_f64(double x) {
#pragma unroll
  for (u32 o = 8; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o, 16);
  return x;
}

// First index i of tl[0..n) with tl[i] >= k, per half (n = 0 for a half that
// does not search).
__device__ __forceinline__ u32 half_lower_bound(const uint16_t* tl, u32 n, u32 k, u32 hl, u32 hb) {
  u32 lo = 0;
  while (__any_sync(kFullMask, n > 16)) {
    const bool big = n > 16;
    const u32 step = (n + 15) >> 4;
    const bool lt = big && hl * step < n && tl[lo + hl * step] < k;
    u32 c = __popc(half_ballot(lt, hb));
    if (big) {
      if (c == 0) c = 1;
      lo += (c - 1) * step;
      n = min(step, n - (c - 1) * step);
    }
  }
  const bool lt = hl < n && tl[lo + hl] < k;
  return lo + __popc(half_ballot(lt, hb));
}

// Inserts k at tl[pos] of a list of n entries for halves with `ins`.
__device__ __forceinline__ void half_insert(uint16_t* tl, u32 n, u32 pos, u32 k, u32 hl, bool ins) {
  u32 top = ins ? n : pos;
  while (__any_sync(kFullMask, top > pos)) {
    const bool go = top > pos;
    const u32 cnt = go ? min(16u, top - pos) : 0u;
    const u32 src = top - 1 - hl;
    const bool a = hl < cnt;
    const uint16_t v = a ? tl[src] : (uint16_t)0;
    __syncwarp();
    if (a) tl[src + 1] = v;
    __syncwarp();
    if (go) top = top > pos + 16 ? top - 16 : pos;
  }
  if (ins && hl == 0) tl[pos] = (uint16_t)k;
  __syncwarp();
}

// Drops the entries of topics with a zero count from tl[0..n) for halves with
// n > 0 (stable, in place) and clears their in-list bits; returns the new
// length.
__device__ __forceinline__ u32 half_compact(uint16_t* tl, u32 n, const uint16_t* cnt, u32* inl, u32 hl, u32 hb) {
  u32 out = 0;
  for (u32 b = 0; __any_sync(kFullMask, b < n); b += 16) {
    const u32 e = b + hl;
    const bool in = e < n;
    const u32 k = in ? (u32)tl[e] : 0u;
    const bool keep = in && cnt[k] != 0;
    const u32 ball = half_ballot(keep, hb);
    __syncwarp();
    if (keep) tl[out + __popc(ball & ((1u << hl) - 1u))] = (uint16_t)k;
    if (in && !keep) atomicAnd(inl + (k >> 5), ~(1u << (k & 31)));
    out += __popc(ball);
    __syncwarp();
  }
  return out;
}

// Counts, sorted topic list and in-list bitmap of the document z[0..L) for
// halves with `build` (Kp topics, a multiple of 64).
__device__ __forceinline__ void half_build(uint16_t* cnt, uint16_t* tl, u32* inl, const u32* z, u32 L, u32 K, u32 Kp,
                                           u32 hl, u32 hb, bool build, u32* status, u32& nz, u32& nl) {
  if (build)
    for (u32 i = hl; i < Kp / 8; i += 16) reinterpret_cast<uint4*>(cnt)[i] = make_uint4(0, 0, 0, 0);
  __syncwarp();
  if (build)
    for (u32 i = hl; i < L; i += 16) {
      u32 k = z[i];
      if (k >= K) {
        *status |= kStatusBadTopic;
        k %= K;
      }
      atomicAdd(reinterpret_cast<u32*>(cnt) + (k >> 1), 1u << ((k & 1) * 16));
    }
  __syncwarp();
  const u32 below = (1u << hl) - 1u;
  u32 pos = 0;
  for (u32 b = 0; b < Kp; b += 16) {
    const bool nzb = build && cnt[b + hl] != 0;
    const u32 msk = half_ballot(nzb, hb);
    if (nzb) tl[pos + __popc(msk & below)] = (uint16_t)(b + hl);
    if (build && hl == 0) {
      if ((b & 31) == 0)
        inl[b >> 5] = msk;
      else
        inl[b >> 5] |= msk << 16;
    }
    pos += __popc(msk);
  }
  __syncwarp();
  if (build) nz = nl = pos;
}

template <bool LL>
__global__ void __launch_bounds__(32 * kHalfWarps, 2) z_sweep_half_kernel(HalfArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  __shared__ unsigned long long blk_stats[4];  // tokens, documents, sparse work, sparse draws
  if (threadIdx.x < 4) blk_stats[threadIdx.x] = 0;
  __syncthreads();
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31;
  const u32 hl = lane & 15, hb = lane & 16;
  unsigned char* sb = zsm + (size_t)(threadIdx.x >> 4) * kHalfSlotStride;
  uint16_t* cnt = reinterpret_cast<uint16_t*>(sb);
  uint16_t* tl = cnt + kHalfMaxK;
  u32* inl = reinterpret_cast<u32*>(tl + kHalfMaxK);
  uint4* stage = reinterpret_cast<uint4*>(inl + kHalfMaxK / 32);
  const u32 K = m.K, V = m.V;
  const u32 Kp = (K + 63) & ~63u;
  const float alpha = m.alpha;
  const u32 t = p.t_dev ? *p.t_dev : p.t;

  // this half's document
  u32 doc = 0, L = 0, basei = 0, nz = 0, nl = 0;
  u64 off = 0;
  bool done = false;
  double ll_acc = 0.0, ll_skip = 0.0;
  u32 status = 0;

  while (true) {
    // halves whose document is finished take the next one
    const bool need = !done && basei >= L;
    if (__any_sync(kFullMask, need)) {
      u32 d = 0;
      if (need && hl == 0) d = atomicAdd(p.work, 1u);
      d = __shfl_sync(kFullMask, d, 0, 16);
      bool build = false;
      if (need) {
        basei = 0;
        if (d >= p.n_docs) {
          done = true;
          L = 0;
        } else {
          doc = p.order ? p.order[d] : d;
          L = p.d_len[doc];
          off = p.d_idx[doc];
          if (L > kHalfMaxDocLen) {
            status |= kStatusDocTooLong;
            L = 0;
          } else if (off + L > p.n_tokens) {
            status |= kStatusDocRange;
            L = 0;
          } else if (L == 0) {  // an empty document: nothing to sweep
            if (hl == 0) {
              if (p.K_d) p.K_d[doc] = 0;
              atomicAdd(blk_stats + 1, 1ull);
            }
          } else {
            build = true;
          }
        }
      }
      half_build(cnt, tl, inl, p.z + (build ? off : 0), build ? L : 0, K, Kp, hl, hb, build, &status, nz, nl);
      continue;
    }
    if (__all_sync(kFullMask, done)) break;

    // one chunk of up to 16 tokens per half
    const u32 nt = done ? 0u : min(16u, L - basei);
    const u32 i = basei + hl;
    const bool valid = hl < nt;
    u32 my_w = valid ? p.w[off + i] : 0u;
    u32 my_z = valid ? p.z[off + i] : 0u;
    if (my_w >= V) {
      status |= kStatusBadWord;
      my_w %= V;
    }
    if (my_z >= K) my_z %= K;
    const U4 r = draw4(p.tok_base + off + i, t, kStreamZ, 0, m.key0, m.key1);
    const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
    const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
    const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
    const u64 my_row = (u64)my_w * K;
    const u64 my_al = (valid && my_nw) ? __ldg(m.al + my_row + my_s) : 0ull;
    __syncwarp();
    stage[2 * hl] = make_uint4(my_z, r.x, r.y, my_nw);
    stage[2 * hl + 1] = make_uint4((u32)my_row, (u32)(my_row >> 32), (u32)my_A, (u32)(my_A >> 32));
    __syncwarp();
    u32 new_z = my_z;
    u32 chunk_st = 0;  // (sum of min(nz without the token, nnz[w])) << 6 + sparse draws
    const u32 ntmax = max(nt, __shfl_xor_sync(kFullMask, nt, 16));
    for (u32 j = 0; j < ntmax; ++j) {
      const bool act = j < nt;
      const uint4 s0 = stage[2 * j], s1 = stage[2 * j + 1];
      const u32 zj = s0.x, r0 = s0.y, r1 = s0.z, nw = act ? s0.w : 0u;
      const u64 row = ((u64)s1.y << 32) | s1.x;
      const u64 Aw = ((u64)s1.w << 32) | s1.z;
      const u32* __restrict__ qrow = m.q + row;
      const u64* __restrict__ crow = m.csr + row;
      // remove the token's current topic
      const u32 cz = act ? (u32)cnt[zj] : 0u;
      __syncwarp();
      if (act && hl == 0) cnt[zj] = (uint16_t)(cz - 1u);
      if (act && cz == 1u) --nz;
      __syncwarp();
      // sparse mass over this lane's contiguous chunk of the shorter list
      const bool word_side = nw < kWordSideFactor * nl;
      const u32 len = act ? (word_side ? nw : nl) : 0u;
      const u32 cper = (len + 15) >> 4;
      const u32 e0 = min(len, hl * cper), e1 = min(len, e0 + cper);
      const u32 n_my = e1 - e0;
      // The first kHalfRegs elements of the chunk keep their masses in
      // registers; the rest are summed in unrolled batches of independent
      // loads (a scalar loop would wait on each gather in turn).
      u32 kk[kHalfRegs], qq[kHalfRegs];
      u64 ms[kHalfRegs];
#pragma unroll
      for (u32 c = 0; c < kHalfRegs; ++c) {
        u32 kx = 0, qx = 0;
        if (c < n_my) {
          if (word_side) {
            const u64 ent = __ldg(crow + e0 + c);
            kx = (u32)ent & 0xffffu;
            qx = (u32)(ent >> 32);
          } else {
            kx = tl[e0 + c];
          }
        }
        kk[c] = kx;
        qq[c] = qx;
      }
#pragma unroll
      for (u32 c = 0; c < kHalfRegs; ++c)
        if (c < n_my && !word_side) qq[c] = __ldg(qrow + kk[c]);
      u64 first = 0;
#pragma unroll
      for (u32 c = 0; c < kHalfRegs; ++c) {
        ms[c] = (u64)cnt[kk[c]] * qq[c];
        first += ms[c];
      }
      u64 ls = first;
      for (u32 b = kHalfRegs; b < n_my; b += kHalfBatch) {
        u32 kb[kHalfBatch], qb[kHalfBatch];
#pragma unroll
        for (u32 c = 0; c < kHalfBatch; ++c) {
          u32 kx = 0, qx = 0;
          if (b + c < n_my) {
            if (word_side) {
              const u64 ent = __ldg(crow + e0 + b + c);
              kx = (u32)ent & 0xffffu;
              qx = (u32)(ent >> 32);
            } else {
              kx = tl[e0 + b + c];
            }
          }
          kb[c] = kx;
          qb[c] = qx;
        }
#pragma unroll
        for (u32 c = 0; c < kHalfBatch; ++c)
          if (b + c < n_my && !word_side) qb[c] = __ldg(qrow + kb[c]);
#pragma unroll
        for (u32 c = 0; c < kHalfBatch; ++c) ls += (u64)cnt[kb[c]] * qb[c];
      }
      const u64 incl = half_incl_scan_u64(ls, hl);
      const u64 B = __shfl_sync(kFullMask, incl, 15, 16);
      int degenerate;
      const int sp = take_sparse(r0, alpha, Aw, B, &degenerate);
      const bool sparse = act && sp && !degenerate;
      // sparse selection: lane f's chunk holds the crossing element; when it
      // lies among lane f's register elements the topic is read from there
      const u64 target = scale_u32(r1, B);
      const u32 f = (__ffs(half_ballot(incl > target, hb)) - 1) & 15u;
      u32 kc = kk[kHalfRegs - 1];
      {
        u64 run = incl - ls;
        bool found = false;
#pragma unroll
        for (u32 c = 0; c + 1 < kHalfRegs; ++c) {
          run += ms[c];
          if (!found && run > target) {
            found = true;
            kc = kk[c];
          }
        }
      }
      u32 k_sp = __shfl_sync(kFullMask, kc, f, 16);
      const u64 pre_f = __shfl_sync(kFullMask, incl - ls, f, 16);
      const u64 first_f = __shfl_sync(kFullMask, first, f, 16);
      // otherwise a second pass over lane f's elements past its registers
      const bool need2 = sparse && pre_f + first_f <= target;
      if (__any_sync(kFullMask, need2)) {
        u64 run = pre_f + first_f;
        const u32 f0 = min(len, f * cper), f1 = min(len, f0 + cper);
        bool found = !need2;
        for (u32 s0e = f0 + kHalfRegs; __any_sync(kFullMask, !found && s0e < f1); s0e += 16) {
          const u32 e = s0e + hl;
          const bool on = !found && e < f1;
          u64 mass = 0;
          u32 kx = 0;
          if (on) {
            u32 qx;
            if (word_side) {
              const u64 ent = __ldg(crow + e);
              kx = (u32)ent & 0xffffu;
              qx = (u32)(ent >> 32);
            } else {
              kx = tl[e];
              qx = __ldg(qrow + kx);
            }
            mass = (u64)cnt[kx] * qx;
          }
          const u64 in2 = half_incl_scan_u64(mass, hl);
          const u64 tot = __shfl_sync(kFullMask, in2, 15, 16);
          const u32 jj = (__ffs(half_ballot(!found && run + in2 > target, hb)) - 1) & 15u;
          const u32 kj = __shfl_sync(kFullMask, kx, jj, 16);
          if (!found) {
            if (run + tot > target) {
              k_sp = kj;
              found = true;
            } else {
              run += tot;
            }
          }
        }
      }
      // dense draw: lane j's alias entry and fourth word
      const u32 r3 = __shfl_sync(kFullMask, r.w, j, 16);
      const u64 ea = __shfl_sync(kFullMask, my_al, j, 16);
      const u32 k_dn = alias_pick(ea, r3);
      const u32 k = degenerate ? zj : (sp ? k_sp : k_dn);
      const u32 nzm = nz;
      // add the new topic
      const u32 ck = act ? (u32)cnt[k] : 1u;
      __syncwarp();
      if (act && hl == 0) cnt[k] = (uint16_t)(ck + 1u);
      bool ins = false;
      if (act && ck == 0u) {
        ++nz;
        ins = !((inl[k >> 5] >> (k & 31)) & 1u);
      }
      if (__any_sync(kFullMask, ins)) {
        const u32 pos = half_lower_bound(tl, ins ? nl : 0u, k, hl, hb);
        half_insert(tl, nl, pos, k, hl, ins);
        if (ins) {
          if (hl == 0) inl[k >> 5] |= 1u << (k & 31);
          ++nl;
        }
        __syncwarp();
      }
      const bool cmp = act && nl - nz > kHalfDead;
      if (__any_sync(kFullMask, cmp)) {
        const u32 n2 = half_compact(tl, cmp ? nl : 0u, cnt, inl, hl, hb);
        if (cmp) nl = n2;
      }
      if (act && hl == 0) {
        atomicAdd(m.n + row + k, 1u);
        chunk_st += (min(nzm, nw) << 6) + (sparse ? 1u : 0u);
      }
      if (act && hl == j) new_z = k;
      __syncwarp();
    }
    if (hl == 0 && nt) {
      atomicAdd(blk_stats + 2, (unsigned long long)(chunk_st >> 6));
      atomicAdd(blk_stats + 3, (unsigned long long)(chunk_st & 63u));
    }
    if (valid) {
      p.z[off + i] = new_z;
      if (LL) {  // log Phi[new topic][word], one token per lane
        const u32 qk = __ldg(m.q + my_row + new_z);
        if (qk)
          ll_acc += log((double)qk) - 22.18070977791825;  // 32 log 2
        else
          ll_skip += 1.0;
      }
    }
    basei += 16;
    // halves whose document ended with this chunk
    const bool fin = nt && basei >= L;
    if (__any_sync(kFullMask, fin)) {
      if (fin && hl == 0 && p.K_d) p.K_d[doc] = nz;
      if (LL) {
        double dl = 0.0;
        if (fin)
          for (u32 e = hl; e < nl; e += 16) {
            const u32 c = cnt[tl[e]];
            if (c) dl += lgamma((double)alpha + (double)c) - a.lg_a;
          }
        dl = half_sum_f64(dl);
        if (fin && hl == 0) ll_acc += dl + a.lg_Ka - lgamma((double)K * (double)alpha + (double)L);
      }
      if (fin && hl == 0) {
        atomicAdd(blk_stats + 0, (unsigned long long)L);
        atomicAdd(blk_stats + 1, 1ull);
      }
    }
  }
  if (LL) {
    ll_acc = warp_sum_f64(ll_acc);
    ll_skip = warp_sum_f64(ll_skip);
    if (lane == 0) {
      atomicAdd(p.ll, ll_acc);
      atomicAdd(p.ll + 1, ll_skip);
    }
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

bool launch_z_sweep_half(const ModelDev& m, const ZLaunch& z, cudaStream_t s) {
  if (m.K > kHalfMaxK) return false;
  if (!z.n_docs) return true;
  HalfArgs a;
  a.m = m;
  a.z = z;
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  const size_t smem = kHalfSlotStride * 2 * kHalfWarps;
  const bool ll = (z.flags & 1u) && z.ll;
  auto kern = ll ? z_sweep_half_kernel<true> : z_sweep_half_kernel<false>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kHalfWarps, smem);
  if (per_sm < 1) per_sm = 1;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (z.n_docs + 2 * kHalfWarps - 1) / (2 * kHalfWarps);
  if (blocks > need) blocks = need;
  kern<<<blocks, 32 * kHalfWarps, smem, s>>>(a);
  return true;
}

}  // namespace gpulda
