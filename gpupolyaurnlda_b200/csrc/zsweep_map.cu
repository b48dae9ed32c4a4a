// zsweep_map.cu -- the z sweep for large K, with each document's topic counts
// in a warp-cooperative Robin Hood hash map held in shared memory (reference:
// the per-document HashMap of src/cu/hashmap.cuh:13-334 used by sample_topics,
// src/cu/topics.cu:36-105; there it lives in the device heap and is rebuilt by
// a retry loop on overflow).
//
// The map is order-preserving: a topic k has home slot floor(k * C / K)
// (monotone in k), collisions are resolved by linear probing with the Robin
// Hood rule (within a run, entries sit in key order, so a larger key yields
// its slot to a smaller one), deletions shift the following displaced entries
// back by one, and a tail of T slots past the C home slots absorbs runs so they
// never wrap.  Reading the slots in order therefore lists the document's topics
// in ascending order, which makes the sparse draw identical to the ascending
// walk of the dense-count kernel and of the CPU oracle.  An entry is
// (topic << 16 | count) in 32 bits; 0xffffffff marks an empty slot.
//
// Capacity per document: C = next power of two >= 2 * min(L, K) (at least 32),
// T = min(L, K) rounded up to 32.  A document holds at most min(L, K) distinct
// topics and every entry sits at or after its home, so an entry's slot is at
// most C - 1 + (entries) < C + T: no run ever passes the end.
#include <algorithm>
#include <cmath>

#include "kernels.cuh"
#include "warp.cuh"

namespace gpulda {

namespace {

constexpr u32 kMaxDocLen = 65535u;
constexpr u32 kEmpty = 0xffffffffu;

struct MapArgs {
  ModelDev m;
  ZLaunch z;
  u32 slots;     // slots per warp (capacity for the longest document of the launch)
  u32 lmax;      // longest document this launch accepts
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

struct DocMap {
  u32* slot;
  u32 C;   // home slots
  u32 S;   // C + tail
  u32 K;
  __device__ __forceinline__ u32 home(u32 k) const { return (u32)(((u64)k * C) / K); }
};

// First slot p >= home(k) that is empty or holds a key >= k; *hit tells
// whether it holds k itself.  Warp-cooperative, 32 slots per round.
__device__ __forceinline__ u32 map_find(const DocMap& mp, u32 k, u32 lane, bool* hit) {
  for (u32 base = mp.home(k); base < mp.S; base += 32) {
    const u32 i = base + lane;
    const u32 e = i < mp.S ? mp.slot[i] : kEmpty;
    const bool stop = e == kEmpty || (e >> 16) >= k;
    const u32 ball = __ballot_sync(kFullMask, stop);
    if (ball) {
      const u32 l = __ffs(ball) - 1;
      const u32 el = __shfl_sync(kFullMask, e, l);
      *hit = el != kEmpty && (el >> 16) == k;
      return base + l;
    }
  }
  *hit = false;
  return mp.S;  // unreachable: capacity rule
}

// First empty slot at or after p.
__device__ __forceinline__ u32 map_next_empty(const DocMap& mp, u32 p, u32 lane) {
  for (u32 base = p; base < mp.S; base += 32) {
    const u32 i = base + lane;
    const bool empty = i >= mp.S || mp.slot[i] == kEmpty;
    const u32 ball = __ballot_sync(kFullMask, empty);
    if (ball) return base + (__ffs(ball) - 1);
  }
  return mp.S;
}

// Count of topic k += 1 (inserting it with count 1 if absent).
__device__ __forceinline__ bool map_add(const DocMap& mp, u32 k, u32 lane) {
  bool hit;
  const u32 p = map_find(mp, k, lane, &hit);
  if (hit) {
    if (lane == 0) mp.slot[p] += 1u;
    __syncwarp();
    return false;
  }
  // shift the run [p, q) one slot right, then place k at p
  const u32 q = map_next_empty(mp, p, lane);
  if (q >= mp.S) return false;  // unreachable under the capacity rule
  for (u32 top = q; top > p; top = top > p + 32 ? top - 32 : p) {
    const u32 src = top - 1 - lane;
    const bool act = lane < top - p;
    const u32 v = act ? mp.slot[src] : 0u;
    __syncwarp();
    if (act) mp.slot[src + 1] = v;
    __syncwarp();
  }
  if (lane == 0) mp.slot[p] = (k << 16) | 1u;
  __syncwarp();
  return true;
}

// Count of topic k (present) -= 1, deleting it when it reaches zero
// (backward shift of the displaced entries that follow).
__device__ __forceinline__ bool map_remove(const DocMap& mp, u32 k, u32 lane) {
  bool hit;
  const u32 p = map_find(mp, k, lane, &hit);
  if (!hit) return false;  // unreachable: the token's topic is counted
  const u32 e = mp.slot[p];
  __syncwarp();
  if ((e & 0xffffu) > 1u) {
    if (lane == 0) mp.slot[p] = e - 1u;
    __syncwarp();
    return false;
  }
  // q = first slot after p that is empty or holds an entry at its home slot
  u32 q = mp.S;
  for (u32 base = p + 1; base < mp.S; base += 32) {
    const u32 i = base + lane;
    const u32 v = i < mp.S ? mp.slot[i] : kEmpty;
    const bool stop = v == kEmpty || mp.home(v >> 16) == i;
    const u32 ball = __ballot_sync(kFullMask, stop);
    if (ball) {
      q = base + (__ffs(ball) - 1);
      break;
    }
  }
  for (u32 b = p + 1; b < q; b += 32) {
    const u32 src = b + lane;
    const u32 v = src < q ? mp.slot[src] : 0u;
    __syncwarp();
    if (src < q) mp.slot[src - 1] = v;
    __syncwarp();
  }
  if (lane == 0) mp.slot[q - 1] = kEmpty;
  __syncwarp();
  return true;
}

__global__ void __launch_bounds__(256, 4) z_sweep_map_kernel(MapArgs a) {
  extern __shared__ __align__(16) unsigned char zsm[];
  const ModelDev& m = a.m;
  const ZLaunch& p = a.z;
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32 K = m.K, V = m.V;
  u32* slots = (u32*)(zsm + (size_t)warp * a.slots * 4);
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
    if (L > kMaxDocLen || L > a.lmax) {
      status |= kStatusDocTooLong;
      continue;
    }
    if (off + L > p.n_tokens) {
      status |= kStatusDocRange;
      continue;
    }
    const u32 dk = min(L, K);
    DocMap mp;
    mp.slot = slots;
    mp.K = K;
    mp.C = max(32u, 1u << (32 - __clz(max(1u, 2 * dk - 1))));
    mp.S = mp.C + ((dk + 31) & ~31u);
    for (u32 i = lane; i < mp.S; i += 32) slots[i] = kEmpty;
    __syncwarp();
    u32 nz = 0;
    for (u32 i = 0; i < L; ++i) {
      u32 k = p.z[off + i];
      if (k >= K) {
        status |= kStatusBadTopic;
        k %= K;
      }
      nz += map_add(mp, k, lane) ? 1u : 0u;
    }
    const u32 cper = mp.S / 32;  // slots per lane (S is a multiple of 32)

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
      // the dense draw's slot in the word's sparse alias table (nnz slots)
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
      const u64 my_al = (valid && my_nw) ? __ldg(m.al + (size_t)my_w * K + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      for (u32 j = 0; j < nt; ++j) {
        const u32 wj = __shfl_sync(kFullMask, my_w, j);
        const u32 zj = __shfl_sync(kFullMask, my_z, j);
        const u32 r0 = __shfl_sync(kFullMask, r.x, j);
        const u32 r1 = __shfl_sync(kFullMask, r.y, j);
        const u64 Aw = __shfl_sync(kFullMask, my_A, j);
        const u32* __restrict__ qrow = m.q + (size_t)wj * K;
        nz -= map_remove(mp, zj, lane) ? 1u : 0u;
        // sparse mass over this lane's contiguous slots (ascending topics)
        u64 ls = 0;
        const u32 s0 = lane * cper;
        for (u32 s = s0; s < s0 + cper; ++s) {
          const u32 e = slots[s];
          if (e != kEmpty) ls += (u64)(e & 0xffffu) * __ldg(qrow + (e >> 16));
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
            for (u32 b0 = f * cper; b0 < f * cper + cper; b0 += 32) {
              const u32 s = b0 + lane;
              u64 mass = 0;
              u32 kk = 0;
              if (s < f * cper + cper) {
                const u32 e = slots[s];
                if (e != kEmpty) {
                  kk = e >> 16;
                  mass = (u64)(e & 0xffffu) * __ldg(qrow + kk);
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
        const u32 nw = __shfl_sync(kFullMask, my_nw, j);
        if (lane == 0) {
          atomicAdd(m.n + (size_t)wj * K + k, 1u);
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
        nz += map_add(mp, k, lane) ? 1u : 0u;
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (valid) p.z[off + i] = new_z;
    }
    if (lane == 0 && p.K_d) p.K_d[doc] = nz;
    if (want_ll) {
      double dl = 0.0;
      for (u32 s = lane; s < mp.S; s += 32) {
        const u32 e = slots[s];
        if (e != kEmpty) dl += lgamma((double)m.alpha + (double)(e & 0xffffu)) - a.lg_a;
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

// Map slots a warp needs for documents of up to lmax tokens.
u32 z_map_slots(u32 K, u32 lmax) {
  const u32 dk = std::min(std::max(lmax, 1u), K);
  u32 C = 32;
  while (C < 2 * dk) C <<= 1;
  return C + ((dk + 31) & ~31u);
}

bool launch_z_sweep_map(const ModelDev& m, const ZLaunch& z, cudaStream_t s, u32 lmax) {
  if (!z.n_docs) return true;
  MapArgs a;
  a.m = m;
  a.z = z;
  a.lmax = lmax;
  a.slots = z_map_slots(m.K, lmax);
  a.lg_a = std::lgamma((double)m.alpha);
  a.lg_Ka = std::lgamma((double)m.K * (double)m.alpha);
  const size_t per_warp = (size_t)a.slots * 4;
  constexpr size_t kBudget = 200 * 1024;
  u32 wpb = 8;
  while (wpb > 1 && per_warp * wpb > kBudget) --wpb;
  if (per_warp * wpb > kBudget) return false;
  const size_t smem = per_warp * wpb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(z_sweep_map_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, z_sweep_map_kernel, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  u32 blocks = (u32)(device_sm_count() * per_sm);
  const u32 need = (z.n_docs + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  z_sweep_map_kernel<<<blocks, 32 * wpb, smem, s>>>(a);
  return true;
}

}  // namespace gpulda
