// kernels.cu -- the sampler's device code for sm_100a.
//
// One iteration (reference: src/cu/train.cu:137-172) is
//   phi_draw      x[k][w] ~ Poisson(beta + n[k][w]); S[k] = sum_w x; n <- 0
//   alias_build   q[w][k] = floor(x * 2^32 / S[k]); A[w] = sum_k q; alias table of
//                 word w over topics with weights q[w][.]
//   doc_offsets   exclusive scan of document lengths
//   z_sweep       per document, sequentially per token: remove z_i, draw
//                 p(k) ~ q[w_i][k] * (alpha + m_dk), add back, n[w_i][z_i] += 1
// All arrays indexed by (word, topic) are word-major: index w*K + k.
#include "kernels.cuh"
#include "warp.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace gpulda {

namespace {

// ---------------------------------------------------------------------------
// Initial counts (reference: polya_urn_init, src/cu/polyaurn.cu:61-79):
// n[w][k] ~ Poisson(beta + floor(C[w] / K)).  One Philox block serves the
// four cells 4g .. 4g+3.
// ---------------------------------------------------------------------------
__global__ void init_counts_kernel(u32* __restrict__ n, u32 K, u32 V, const u32* __restrict__ C, PoisTables tb,
                                   double beta, u32 key0, u32 key1) {
  const u64 cells = (u64)K * V;
  const u64 groups = (cells + 3) / 4;
  for (u64 gi = (u64)blockIdx.x * blockDim.x + threadIdx.x; gi < groups; gi += (u64)gridDim.x * blockDim.x) {
    const U4 r = draw4(gi, 0, kStreamInitCounts, 0, key0, key1);
#pragma unroll
    for (u32 u = 0; u < 4; ++u) {
      const u64 c = gi * 4 + u;
      if (c < cells) {
        const u32 lam_n = C[c / K] / K;
        n[c] = poisson_draw(lam_n, beta, u4_word(r, u), c, 0, kStreamInitCounts, key0, key1, tb);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Phi draw (reference: polya_urn_sample + draw_poisson + polya_urn_reset,
// src/cu/polyaurn.cu:7-36,87-141).  Each block owns a contiguous range of
// rows; threads take groups of four cells (one Philox block, 16-byte loads and
// stores when the group lies inside the range).  Per-topic sums are gathered
// in shared memory (integer atomics: order-free) and flushed once per block.
// ---------------------------------------------------------------------------
// Cells [c0, c1) of one model (local cell indices; n and q point at its cell
// 0).  Nonzero draws are added to the per-topic sums: into shared memory when
// s_sum is given, else straight into S.
__device__ __forceinline__ void phi_rows(u32 K, u64 c0, u64 c1, u32* __restrict__ n, u32* __restrict__ q, u64* S,
                                         const PoisTables& tb, double beta, u32 key0, u32 key1, u32 t,
                                         unsigned long long* s_sum) {
  for (u64 gi = c0 / 4 + threadIdx.x; gi * 4 < c1; gi += blockDim.x) {
    const u64 cb = gi * 4;
    const U4 r = draw4(gi, t, kStreamPhi, 0, key0, key1);
    const bool whole = cb >= c0 && cb + 4 <= c1;
    u32 nv[4];
    if (whole) {
      const uint4 v = *reinterpret_cast<const uint4*>(n + cb);
      nv[0] = v.x;
      nv[1] = v.y;
      nv[2] = v.z;
      nv[3] = v.w;
    } else {
#pragma unroll
      for (u32 u = 0; u < 4; ++u) nv[u] = (cb + u >= c0 && cb + u < c1) ? n[cb + u] : 0u;
    }
    u32 xv[4];
#pragma unroll
    for (u32 u = 0; u < 4; ++u) xv[u] = poisson_draw(nv[u], beta, u4_word(r, u), cb + u, t, kStreamPhi, key0, key1, tb);
    if (whole) {
      *reinterpret_cast<uint4*>(q + cb) = make_uint4(xv[0], xv[1], xv[2], xv[3]);
      *reinterpret_cast<uint4*>(n + cb) = make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (u32 u = 0; u < 4; ++u) {
      const u64 c = cb + u;
      if (c < c0 || c >= c1) continue;
      if (!whole) {
        q[c] = xv[u];
        n[c] = 0;
      }
      if (xv[u]) {
        const u32 k = (u32)(c % K);
        if (s_sum)
          atomicAdd(&s_sum[k], (unsigned long long)xv[u]);
        else
          atomicAdd((unsigned long long*)&S[k], (unsigned long long)xv[u]);
      }
    }
  }
}

// Four blocks per SM: the rejection sampler's registers otherwise held the
// kernel to two (1.4x faster at K=10000; its spills are on the rare path).
__global__ void __launch_bounds__(256, 4) phi_draw_kernel(ModelDev m, u32 t, u32 rows_per_block, int smem_sums) {
  extern __shared__ unsigned long long s_sum[];
  const u32 K = m.K;
  if (smem_sums) {
    for (u32 k = threadIdx.x; k < K; k += blockDim.x) s_sum[k] = 0;
    __syncthreads();
  }
  const u32 w0 = blockIdx.x * rows_per_block;
  const u32 w1 = min(m.V, w0 + rows_per_block);
  phi_rows(K, (u64)w0 * K, (u64)w1 * K, m.n, m.q, m.S, m.tables, (double)m.beta, m.key0, m.key1, t,
           smem_sums ? s_sum : nullptr);
  if (smem_sums) {
    __syncthreads();
    for (u32 k = threadIdx.x; k < K; k += blockDim.x)
      if (s_sum[k]) atomicAdd((unsigned long long*)&m.S[k], s_sum[k]);
  }
}

// Phi draw for K a multiple of 4 (the common case): block (bx, by) draws rows
// [bx * rows, (bx + 1) * rows) of topics [1024 by, 1024 (by + 1)); thread i
// owns the four topics 1024 by + 4 i .. + 3 for every row of the block, so its
// 16-byte loads and stores of consecutive threads are contiguous, and it keeps
// the four per-topic sums in registers across the rows: the normalisers need
// no shared memory and one 64-bit atomic per (block, topic) at the end.  Cell
// c = w K + k uses word c & 3 of Philox block c >> 2, exactly as phi_rows, so
// the draws are the same.
// Rows whose counts each thread loads before drawing any of them: the draw of
// a row waits on its 16-byte load, so loads of several rows in flight hide
// the memory latency one row at a time would expose.  With four rows the loop
// needs about 120 registers (two 256-thread blocks per SM); at 64 registers it
// spilled (mid corpus: 1.75 TB/s of its 12 B per cell against 1.51 TB/s with
// one row at a time and four blocks per SM).
constexpr u32 kPhiRowsInFlight = 4;

__global__ void __launch_bounds__(256, 2) phi_draw_cols_kernel(ModelDev m, u32 t, u32 rows_per_block) {
  const u32 K = m.K;
  const u32 k0 = blockIdx.y * 1024u + 4u * threadIdx.x;
  if (k0 >= K) return;
  const u32 w0 = blockIdx.x * rows_per_block;
  const u32 w1 = min(m.V, w0 + rows_per_block);
  const double beta = (double)m.beta;
  // Most cells hold no tokens, and for n = 0 the inversion returns 0 exactly
  // when the cell's word is below the table's first CDF entry: that entry in
  // a register answers those cells without the guide and CDF loads (K=10000:
  // 4.06 against 3.86 TB/s; no difference at K=1000).
  const u32 cdf00 = __ldg(m.tables.cdf);
  u64 acc[4] = {0, 0, 0, 0};
  for (u32 wb = w0; wb < w1; wb += kPhiRowsInFlight) {
    uint4 v[kPhiRowsInFlight];
#pragma unroll
    for (u32 i = 0; i < kPhiRowsInFlight; ++i)
      v[i] = wb + i < w1 ? *reinterpret_cast<const uint4*>(m.n + (u64)(wb + i) * K + k0) : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (u32 i = 0; i < kPhiRowsInFlight; ++i) {
      if (wb + i >= w1) break;
      const u64 cb = (u64)(wb + i) * K + k0;
      const U4 r = draw4(cb >> 2, t, kStreamPhi, 0, m.key0, m.key1);
      const u32 nv[4] = {v[i].x, v[i].y, v[i].z, v[i].w};
      u32 xv[4];
#pragma unroll
      for (u32 u = 0; u < 4; ++u) {
        const u32 ru = u4_word(r, u);
        xv[u] = (nv[u] == 0 && ru < cdf00)
                    ? 0u
                    : poisson_draw(nv[u], beta, ru, cb + u, t, kStreamPhi, m.key0, m.key1, m.tables);
        acc[u] += xv[u];
      }
      *reinterpret_cast<uint4*>(m.q + cb) = make_uint4(xv[0], xv[1], xv[2], xv[3]);
      *reinterpret_cast<uint4*>(m.n + cb) = make_uint4(0, 0, 0, 0);
    }
  }
#pragma unroll
  for (u32 u = 0; u < 4; ++u)
    if (acc[u]) atomicAdd((unsigned long long*)&m.S[k0 + u], (unsigned long long)acc[u]);
}

// Batched Phi draw: block b draws rows [w0, w1) (problem-local word ids) of
// problem p, with (p, w0, w1) from the block table.
__global__ void __launch_bounds__(256) phi_draw_batch_kernel(ModelDev ar, BatchPhiDev bp, const u32* t_dev) {
  extern __shared__ unsigned long long s_sum[];
  const uint4 e = bp.blocks[blockIdx.x];
  const u32 pb = e.x, K = bp.K[pb];
  for (u32 k = threadIdx.x; k < K; k += blockDim.x) s_sum[k] = 0;
  __syncthreads();
  const u64 cell0 = bp.cell_base[pb];
  PoisTables tb{bp.cdf + (size_t)pb * kPoisN * kPoisW, bp.guide + (size_t)pb * kPoisN * 256, bp.lfac + (size_t)pb * kLogFacN};
  u64* S = ar.S + bp.S_off[pb];
  phi_rows(K, (u64)e.y * K, (u64)e.z * K, ar.n + cell0, ar.q + cell0, S, tb, (double)bp.beta[pb], bp.key0[pb],
           bp.key1[pb], *t_dev, s_sum);
  __syncthreads();
  for (u32 k = threadIdx.x; k < K; k += blockDim.x)
    if (s_sum[k]) atomicAdd((unsigned long long*)&S[k], s_sum[k]);
}

// ---------------------------------------------------------------------------
// Deterministic parallel alias construction over n items with integer weights
// (reference: build_alias, src/cu/spalias.cu:88-174, which uses atomic work
// queues).  Slot capacity is A = sum_i q_i; item i carries w_i = n*q_i.
// Items with w_i < A are light, the rest heavy, each list in item order.
// The result equals the sequential sweep in which the front heavy fills the
// next light and, on falling below A, is itself filled by the following
// heavy before any further light.  With D_i the exclusive prefix of light
// deficits (A - w) and E_j the inclusive prefix of heavy excesses (w - A):
//   light i  -> alias = heavy j* = min{j : E_j >= D_i}, threshold w_i / A;
//   heavy j with E_j < D_total -> alias = heavy j+1, kept weight
//               A - (D_i + d_i - E_j) with i the light whose deficit interval
//               [D_i, D_i + d_i) contains E_j;
//   other heavies keep the whole slot.
// Every quantity is an exact integer (n <= K <= 32768 keeps n*A below 2^63).
// Entry of item i: threshold | key[i] << 32 | key[alias item] << 48.
// wq[n] holds the weights, key[n] the items' topics; vals[n], idx[n] scratch.
// Block-cooperative.
// ---------------------------------------------------------------------------
__device__ void alias_build_block(const u64* ent, u32 n, u64 A, u64* vals, uint16_t* idx, u64* out, u64* sh) {
  const u32 NT = blockDim.x, tid = threadIdx.x;
  const u32 chunk = (n + NT - 1) / NT;
  const u32 i0 = min(n, tid * chunk), i1 = min(n, i0 + chunk);
  u64 nl = 0, dl = 0, nh = 0, eh = 0;
  for (u32 i = i0; i < i1; ++i) {
    const u64 wi = (u64)n * (ent[i] >> 32);
    if (wi < A) {
      ++nl;
      dl += A - wi;
    } else {
      ++nh;
      eh += wi - A;
    }
  }
  u64 nL, Dtot, nH, Etot;
  u64 ol = block_excl_scan_u64(nl, sh, &nL);
  u64 od = block_excl_scan_u64(dl, sh, &Dtot);
  u64 oh = block_excl_scan_u64(nh, sh, &nH);
  u64 oe = block_excl_scan_u64(eh, sh, &Etot);
  for (u32 i = i0; i < i1; ++i) {
    const u64 wi = (u64)n * (ent[i] >> 32);
    if (wi < A) {
      vals[ol] = od;
      idx[ol] = (uint16_t)i;
      od += A - wi;
      ++ol;
    } else {
      oe += wi - A;
      vals[nL + oh] = oe;
      idx[nL + oh] = (uint16_t)i;
      ++oh;
    }
  }
  __syncthreads();
  const u64* Ev = vals + nL;
  const uint16_t* Hi = idx + nL;
  auto key = [&](u32 i) -> u64 { return ent[i] & 0xffffu; };
  for (u32 i = tid; i < (u32)nL; i += NT) {
    const u64 D = vals[i];
    u32 lo = 0, hi = (u32)nH - 1;  // first j with E_j >= D (exists: D < Dtot = E_last)
    while (lo < hi) {
      const u32 mid = (lo + hi) >> 1;
      if (Ev[mid] >= D) hi = mid; else lo = mid + 1;
    }
    const u32 l = idx[i];
    out[l] = (key(Hi[lo]) << 48) | (key(l) << 32) | alias_threshold((u64)n * (ent[l] >> 32), A);
  }
  for (u32 j = tid; j < (u32)nH; j += NT) {
    const u32 h = Hi[j];
    const u64 E = Ev[j];
    if (E < Dtot) {
      u32 lo = 0, hi = (u32)nL - 1;  // last i with D_i <= E (D_0 = 0)
      while (lo < hi) {
        const u32 mid = (lo + hi + 1) >> 1;
        if (vals[mid] <= E) lo = mid; else hi = mid - 1;
      }
      const u64 d = A - (u64)n * (ent[idx[lo]] >> 32);
      const u64 over = vals[lo] + d - E;
      out[h] = (key(Hi[j + 1]) << 48) | (key(h) << 32) | alias_threshold(A - over, A);
    } else {
      out[h] = (key(h) << 48) | (key(h) << 32) | 0xffffffffu;
    }
  }
}

// Per word: q = floor(x * 2^32 / S[k]) (clamped) written back densely; the
// word's topics with q > 0 compacted in ascending order into its list
// (q << 32 | k, which is also the alias build's input), the dense mass A, nnz,
// and the sparse alias table over the list.  The dense pass gives each thread
// kPerThread consecutive topics per tile, so a tile needs one block scan.
// The alias build's scratch (10 bytes per nonzero) is shared memory when the
// word's nonzeros fit smem_items, else the block's slice of global scratch.
constexpr u32 kPerThread = 8;

__device__ __forceinline__ void alias_word(u32 K, u32* __restrict__ qrow, const u64* __restrict__ S,
                                           const u64* __restrict__ Sinv, u64* alrow, u64* csrrow, u64* A_out,
                                           u32* nnz_out, u64* s_vals, uint16_t* s_idx, u32 smem_items, u64* g_vals,
                                           uint16_t* g_idx, u64* sh) {
  u64 part = 0, nz = 0;
  const u32 tile = blockDim.x * kPerThread;
  for (u32 t0 = 0; t0 < K; t0 += tile) {
    const u32 k0 = t0 + threadIdx.x * kPerThread;
    u32 qv[kPerThread];
    u32 cnt = 0;
#pragma unroll
    for (u32 c = 0; c < kPerThread; ++c) {
      const u32 k = k0 + c;
      u64 qq = 0;
      if (k < K) {
        const u32 x = qrow[k];
        if (x) {  // a zero count is already a zero q
          const u64 num = (u64)x << 32, sk = S[k];
          if (Sinv) {
            // floor(num / sk) from the reciprocal: the multiply-high is at
            // most 2 below the quotient
            qq = __umul64hi(num, Sinv[k]);
            u64 r = num - qq * sk;
            if (r >= sk) {
              ++qq;
              r -= sk;
            }
            if (r >= sk) ++qq;
          } else {
            qq = num / sk;
          }
          if (qq > 0xffffffffULL) qq = 0xffffffffULL;
          qrow[k] = (u32)qq;
        }
      }
      qv[c] = (u32)qq;
      cnt += qq != 0;
      part += qq;
    }
    u64 tot;
    u64 pos = nz + block_excl_scan_u64(cnt, sh, &tot);
#pragma unroll
    for (u32 c = 0; c < kPerThread; ++c)
      if (qv[c]) csrrow[pos++] = ((u64)qv[c] << 32) | (k0 + c);
    nz += tot;
  }
  const u64 A = block_sum_u64(part, sh);  // (also orders the list writes before the build)
  const u32 n = (u32)nz;
  if (n) {
    const bool in_smem = n <= smem_items;
    alias_build_block(csrrow, n, A, in_smem ? s_vals : g_vals, in_smem ? s_idx : g_idx, alrow, sh);
  }
  if (threadIdx.x == 0) {
    *A_out = A;
    *nnz_out = n;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) alias_build_kernel(ModelDev m, unsigned char* gscratch, size_t slice,
                                                          u32 smem_items) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ u64 sh[33];
  const u32 K = m.K;
  u64* s_vals = (u64*)s_raw;
  uint16_t* s_idx = (uint16_t*)(s_vals + smem_items);
  u64* g_vals = gscratch ? (u64*)(gscratch + (size_t)blockIdx.x * slice) : nullptr;
  uint16_t* g_idx = gscratch ? (uint16_t*)(g_vals + K) : nullptr;
  for (u32 w = blockIdx.x; w < m.V; w += gridDim.x) {
    const size_t row = (size_t)w * K;
    alias_word(K, m.q + row, m.S, m.Sinv, m.al + row, m.csr + row, m.A + w, m.nnz + w, s_vals, s_idx, smem_items,
               g_vals, g_idx, sh);
  }
}

// Batched alias build over global words [w0, w1) of any problems; shared
// memory sized for the largest K among them.
__global__ void __launch_bounds__(256) alias_build_batch_kernel(ModelDev ar, BatchPhiDev bp, u32 Kmax, u32 w0, u32 w1) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ u64 sh[33];
  u64* vals = (u64*)s_raw;
  uint16_t* idx = (uint16_t*)(vals + Kmax);
  for (u32 w = w0 + blockIdx.x; w < w1; w += gridDim.x) {
    const u32 pb = bp.wpid[w], K = bp.K[pb];
    const size_t row = bp.row_off[w];
    alias_word(K, ar.q + row, ar.S + bp.S_off[pb], nullptr, ar.al + row, ar.csr + row, ar.A + w, ar.nnz + w, vals,
               idx, Kmax, nullptr, nullptr, sh);
  }
}

// Reciprocals of the per-topic normalisers, inv[k] = floor((2^64 - 1) / S[k])
// (0 for an empty topic): the alias build then divides by a multiply-high and
// at most two corrections instead of a 64-bit division per nonzero cell.
__global__ void topic_recip_kernel(const u64* __restrict__ S, u64* __restrict__ inv, u32 K) {
  const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < K) {
    const u64 sk = S[k];
    inv[k] = sk ? ~0ull / sk : 0ull;
  }
}

// Advances a device-side iteration counter (replayed graphs read it).
__global__ void bump_kernel(u32* t) { *t += 1; }

__global__ void debug_alias_kernel(const u32* q, u32 K, u64* out) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ u64 sh[33];
  u64* ent = (u64*)s_raw;  // (q << 32 | item)
  u64* vals = ent + K;
  uint16_t* idx = (uint16_t*)(vals + K);
  u64 part = 0;
  for (u32 k = threadIdx.x; k < K; k += blockDim.x) {
    ent[k] = ((u64)q[k] << 32) | k;
    part += q[k];
  }
  const u64 A = block_sum_u64(part, sh);
  alias_build_block(ent, K, A, vals, idx, out, sh);
}

// ---------------------------------------------------------------------------
// Document offsets (reference: compute_d_idx, src/cu/topics.cu:5-32).
// One block; each thread scans a contiguous chunk.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) doc_offsets_kernel(const u32* __restrict__ d_len, u32* __restrict__ d_idx,
                                                           u32 n_docs) {
  __shared__ u64 sh[33];
  const u32 chunk = (n_docs + blockDim.x - 1) / blockDim.x;
  const u32 i0 = min(n_docs, threadIdx.x * chunk), i1 = min(n_docs, i0 + chunk);
  u64 s = 0;
  for (u32 i = i0; i < i1; ++i) s += d_len[i];
  u64 total;
  u64 off = block_excl_scan_u64(s, sh, &total);
  for (u32 i = i0; i < i1; ++i) {
    // Saturate instead of wrapping: buffers hold fewer than 2^32 tokens, so an
    // offset of 2^32 - 1 fails the sweep's range check (offset + length must
    // not pass n_tokens) and is reported, where a wrapped offset could pass it.
    d_idx[i] = off < 0xffffffffull ? (u32)off : 0xffffffffu;
    off += d_len[i];
  }
}

// ---------------------------------------------------------------------------
// Count rebuild n[w][z] += 1 over a token range (reference: the atomicAdd per
// token at the end of sample_topics, src/cu/topics.cu:95).  Tokens are read
// four at a time (16-byte loads of w and z); per load slot the warp groups
// lanes whose tokens hit the same cell (__match_any_sync) and the group's
// lowest lane adds the group's size: one atomic per distinct cell per warp
// step instead of one per token.  Topics >= K and words >= V are reported
// and counted modulo K / V, like the sweeps.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) count_rebuild_kernel(u32* __restrict__ n, const u32* __restrict__ w,
                                                            const u32* __restrict__ z, u64 n_tokens, u32 K, u32 V,
                                                            u32* status) {
  const u32 lane = threadIdx.x & 31;
  const u64 groups = (n_tokens + 3) / 4;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  u32 st = 0;
  // warp-uniform trip count: every lane of a warp takes the same number of steps
  const u64 g0 = (u64)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
  for (u64 gb = g0; gb < groups; gb += stride) {
    const u64 gi = gb + lane;
    u32 wv[4] = {0, 0, 0, 0}, zv[4] = {0, 0, 0, 0};
    u32 nv = 0;  // tokens of this group
    if (gi < groups) {
      const u64 t0 = gi * 4;
      nv = (u32)(n_tokens - t0 < 4 ? n_tokens - t0 : 4);
      if (nv == 4) {
        const uint4 a = *reinterpret_cast<const uint4*>(w + t0);
        const uint4 b = *reinterpret_cast<const uint4*>(z + t0);
        wv[0] = a.x, wv[1] = a.y, wv[2] = a.z, wv[3] = a.w;
        zv[0] = b.x, zv[1] = b.y, zv[2] = b.z, zv[3] = b.w;
      } else {
        for (u32 u = 0; u < nv; ++u) {
          wv[u] = w[t0 + u];
          zv[u] = z[t0 + u];
        }
      }
    }
#pragma unroll
    for (u32 u = 0; u < 4; ++u) {
      const bool on = u < nv;
      u32 wu = wv[u], zu = zv[u];
      if (on && wu >= V) {
        st |= kStatusBadWord;
        wu %= V;
      }
      if (on && zu >= K) {
        st |= kStatusBadTopic;
        zu %= K;
      }
      // lanes without a token get distinct keys that match no cell
      const u64 cell = on ? (u64)wu * K + zu : ~(u64)lane;
      const u32 peers = __match_any_sync(kFullMask, cell);
      if (on && lane == (u32)(__ffs(peers) - 1)) atomicAdd(n + cell, (u32)__popc(peers));
    }
  }
  st = __reduce_or_sync(kFullMask, st);
  if (lane == 0 && st) atomicOr(status, st);
}

__global__ void debug_philox_kernel(const u32* ctr, u32 n, u32 k0, u32 k1, u32* out) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U4 r = philox4x32_10(U4{ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]}, k0, k1);
  out[4 * i] = r.x;
  out[4 * i + 1] = r.y;
  out[4 * i + 2] = r.z;
  out[4 * i + 3] = r.w;
}

__global__ void debug_poisson_kernel(ModelDev m, const u32* count, const u64* idx, u32 n, u32 t, u32 stream,
                                     u32 k0, u32 k1, u32* out) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U4 r = draw4(idx[i] >> 2, t, stream, 0, k0, k1);
  out[i] = poisson_draw(count[i], (double)m.beta, u4_word(r, (u32)(idx[i] & 3)), idx[i], t, stream, k0, k1,
                        m.tables);
}

}  // namespace

static u32 alias_threads(u32 K);
static size_t alias_scratch_item_bytes(u32 n);

int device_sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
  }
  return sms;
}

void launch_init_counts(const ModelDev& m, const u32* C, cudaStream_t s) {
  launch_init_counts_raw(m.n, m.K, m.V, C, m.tables, m.beta, m.key0, m.key1, s);
}

void launch_init_counts_raw(u32* n, u32 K, u32 V, const u32* C, const PoisTables& tb, float beta, u32 key0, u32 key1,
                            cudaStream_t s) {
  const u64 groups = ((u64)K * V + 3) / 4;
  const u32 blocks = (u32)std::max<u64>(1, std::min<u64>((groups + 255) / 256, (u64)device_sm_count() * 16));
  init_counts_kernel<<<blocks, 256, 0, s>>>(n, K, V, C, tb, (double)beta, key0, key1);
}

void launch_phi_draw_batch(const ModelDev& ar, const BatchPhiDev& bp, u32 n_blocks, u32 Kmax, const u32* t_dev,
                           cudaStream_t s) {
  if (!n_blocks) return;
  const size_t smem = (size_t)Kmax * 8;
  if (smem > 48 * 1024) cudaFuncSetAttribute(phi_draw_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  phi_draw_batch_kernel<<<n_blocks, 256, smem, s>>>(ar, bp, t_dev);
}

void launch_alias_build_batch(const ModelDev& ar, const BatchPhiDev& bp, u32 Kmax, u32 w0, u32 w1, cudaStream_t s) {
  if (w1 <= w0) return;
  const u32 nt = alias_threads(Kmax);
  const size_t need = alias_scratch_item_bytes(Kmax);
  if (need > 48 * 1024) cudaFuncSetAttribute(alias_build_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, alias_build_batch_kernel, nt, need);
  if (per_sm < 1) per_sm = 1;
  const u32 blocks = std::min<u32>(w1 - w0, (u32)(device_sm_count() * per_sm * 4));
  alias_build_batch_kernel<<<blocks, nt, need, s>>>(ar, bp, Kmax, w0, w1);
}

void launch_bump(u32* t, cudaStream_t s) { bump_kernel<<<1, 1, 0, s>>>(t); }

void launch_phi_draw(const ModelDev& m, u32 t, cudaStream_t s) {
  if (m.K % 4 == 0) {
    // rows per block: about 64 Ki cells per block, at least 8 rows
    const u32 tiles = (m.K + 1023) / 1024;
    const u32 rows = std::max<u32>(8u, 65536u / std::min<u32>(m.K, 1024u));
    const dim3 grid((m.V + rows - 1) / rows, tiles);
    phi_draw_cols_kernel<<<grid, 256, 0, s>>>(m, t, rows);
    return;
  }
  const u32 rows = std::max<u32>(1u, 65536u / m.K);
  const u32 blocks = (m.V + rows - 1) / rows;
  const int smem_sums = m.K <= 8192;
  const size_t smem = smem_sums ? (size_t)m.K * 8 : 0;
  if (smem > 48 * 1024) cudaFuncSetAttribute(phi_draw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  phi_draw_kernel<<<blocks, 256, smem, s>>>(m, t, rows, smem_sums);
}

static u32 alias_threads(u32 K) {
  u32 nw = (K + 255) / 256;
  if (nw < 1) nw = 1;
  if (nw > 8) nw = 8;
  return 32 * nw;
}

// Alias-build scratch for n items: vals (u64) then idx (u16), 16-byte rounded.
static size_t alias_scratch_item_bytes(u32 n) { return ((size_t)n * 10 + 15) & ~(size_t)15; }

// Items whose scratch the solo alias kernel keeps in shared memory; words with
// more nonzeros use the block's slice of global scratch.  Small shared memory
// keeps several blocks resident per SM at any K.
constexpr u32 kAliasSmemItems = 2048;
constexpr u32 kAliasBlocksPerSm = 4;

static size_t alias_slice_bytes(u32 K) { return (alias_scratch_item_bytes(K) + 255) & ~(size_t)255; }

size_t alias_build_scratch_bytes(u32 K) {
  if (K <= kAliasSmemItems) return 0;
  return alias_slice_bytes(K) * (size_t)device_sm_count() * kAliasBlocksPerSm;
}

void launch_alias_build(const ModelDev& m, cudaStream_t s, void* scratch, size_t scratch_bytes) {
  if (m.Sinv) topic_recip_kernel<<<(m.K + 255) / 256, 256, 0, s>>>(m.S, m.Sinv, m.K);
  const u32 nt = alias_threads(m.K);
  const u32 items = std::min(m.K, kAliasSmemItems);
  const size_t smem = alias_scratch_item_bytes(items);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, alias_build_kernel, nt, smem);
  if (per_sm < 1) per_sm = 1;
  u32 blocks = std::min<u32>(m.V, (u32)(device_sm_count() * per_sm * (m.K <= kAliasSmemItems ? 4 : 1)));
  if (m.K > kAliasSmemItems) {
    const size_t slice = alias_slice_bytes(m.K);
    blocks = std::min<u32>(blocks, (u32)(scratch_bytes / slice));
    if (!blocks) return;  // no scratch: the caller allocates alias_build_scratch_bytes(K)
    alias_build_kernel<<<blocks, nt, smem, s>>>(m, (unsigned char*)scratch, slice, items);
  } else {
    alias_build_kernel<<<blocks, nt, smem, s>>>(m, nullptr, 0, items);
  }
}

void launch_count_rebuild(u32* n, const u32* w, const u32* z, u64 n_tokens, u32 K, u32 V, u32* status,
                          cudaStream_t s) {
  if (!n_tokens) return;
  const u64 groups = (n_tokens + 3) / 4;
  const u32 blocks = (u32)std::max<u64>(1, std::min<u64>((groups + 255) / 256, (u64)device_sm_count() * 8));
  count_rebuild_kernel<<<blocks, 256, 0, s>>>(n, w, z, n_tokens, K, V, status);
}

void launch_doc_offsets(const u32* d_len, u32* d_idx, u32 n_docs, cudaStream_t s) {
  if (!n_docs) return;
  doc_offsets_kernel<<<1, 1024, 0, s>>>(d_len, d_idx, n_docs);
}

void launch_debug_philox(const u32* ctr, u32 n, u32 k0, u32 k1, u32* out, cudaStream_t s) {
  if (!n) return;
  debug_philox_kernel<<<(n + 127) / 128, 128, 0, s>>>(ctr, n, k0, k1, out);
}

void launch_debug_poisson(const ModelDev& m, const u32* count, const u64* idx, u32 n, u32 t, u32 stream,
                          u32 k0, u32 k1, u32* out, cudaStream_t s) {
  if (!n) return;
  debug_poisson_kernel<<<(n + 127) / 128, 128, 0, s>>>(m, count, idx, n, t, stream, k0, k1, out);
}

void launch_debug_alias(const u32* q, u32 K, u64* out, cudaStream_t s) {
  const size_t need = (size_t)K * 8 + alias_scratch_item_bytes(K);
  if (need > 48 * 1024) cudaFuncSetAttribute(debug_alias_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
  debug_alias_kernel<<<1, alias_threads(K), need, s>>>(q, K, out);
}

}  // namespace gpulda
