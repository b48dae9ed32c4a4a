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

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace gpulda {

namespace {

constexpr u32 kMaxDocLen = 65535u;

__device__ __forceinline__ u64 warp_incl_scan_u64(u64 x, u32 lane) {
#pragma unroll
  for (u32 o = 1; o < 32; o <<= 1) {
    const u64 y = __shfl_up_sync(kFullMask, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ u64 warp_sum_u64(u64 x) {
#pragma unroll
  for (u32 o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
  return x;
}

__device__ __forceinline__ double warp_sum_f64(double x) {
#pragma unroll
  for (u32 o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
  return x;
}

// Block-wide exclusive scan of one u64 per thread; `sh` holds 33 entries.
__device__ __forceinline__ u64 block_excl_scan_u64(u64 v, u64* sh, u64* total) {
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const u64 incl = warp_incl_scan_u64(v, lane);
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    u64 x = lane < nw ? sh[lane] : 0;
    x = warp_incl_scan_u64(x, lane);
    sh[lane] = x;
  }
  __syncthreads();
  const u64 off = warp ? sh[warp - 1] : 0;
  *total = sh[nw - 1];
  __syncthreads();
  return off + incl - v;
}

__device__ __forceinline__ u64 block_sum_u64(u64 v, u64* sh) {
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum_u64(v);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  u64 t = 0;
  for (u32 i = 0; i < nw; ++i) t += sh[i];
  __syncthreads();
  return t;
}

// ---------------------------------------------------------------------------
// Initial counts (reference: polya_urn_init, src/cu/polyaurn.cu:61-79):
// n[w][k] ~ Poisson(beta + floor(C[w] / K)).
// ---------------------------------------------------------------------------
__global__ void init_counts_kernel(ModelDev m, const u32* __restrict__ C) {
  const u64 cells = (u64)m.K * m.V;
  for (u64 c = (u64)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += (u64)gridDim.x * blockDim.x) {
    const u32 w = (u32)(c / m.K);
    const u32 lam_n = C[w] / m.K;
    const U4 r = draw4(c, 0, kStreamInitCounts, 0, m.key0, m.key1);
    m.n[c] = poisson_draw(lam_n, (double)m.beta, r, c, 0, kStreamInitCounts, m.key0, m.key1, m.tables);
  }
}

// ---------------------------------------------------------------------------
// Phi draw (reference: polya_urn_sample + draw_poisson + polya_urn_reset,
// src/cu/polyaurn.cu:7-36,87-141).  Each block owns a contiguous range of
// rows; threads stride over its cells (coalesced for any K).  Per-topic sums
// are gathered in shared memory (integer atomics: order-free) and flushed once
// per block.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) phi_draw_kernel(ModelDev m, u32 t, u32 rows_per_block, int smem_sums) {
  extern __shared__ unsigned long long s_sum[];
  const u32 K = m.K;
  if (smem_sums) {
    for (u32 k = threadIdx.x; k < K; k += blockDim.x) s_sum[k] = 0;
    __syncthreads();
  }
  const u32 w0 = blockIdx.x * rows_per_block;
  const u32 w1 = min(m.V, w0 + rows_per_block);
  const u64 c0 = (u64)w0 * K, c1 = (u64)w1 * K;
  const double beta = (double)m.beta;
  for (u64 c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const u32 nk = m.n[c];
    const U4 r = draw4(c, t, kStreamPhi, 0, m.key0, m.key1);
    const u32 x = poisson_draw(nk, beta, r, c, t, kStreamPhi, m.key0, m.key1, m.tables);
    m.q[c] = x;
    m.n[c] = 0;
    if (x) {
      const u32 k = (u32)(c % K);
      if (smem_sums)
        atomicAdd(&s_sum[k], (unsigned long long)x);
      else
        atomicAdd((unsigned long long*)&m.S[k], (unsigned long long)x);
    }
  }
  if (smem_sums) {
    __syncthreads();
    for (u32 k = threadIdx.x; k < K; k += blockDim.x)
      if (s_sum[k]) atomicAdd((unsigned long long*)&m.S[k], s_sum[k]);
  }
}

// ---------------------------------------------------------------------------
// Deterministic parallel alias construction over one row of integer weights
// (reference: build_alias, src/cu/spalias.cu:88-174, which uses atomic work
// queues).  Slot capacity is A = sum_k q_k; item k carries w_k = K*q_k.
// Items with w_k < A are light, the rest heavy, each list in ascending k.
// The result equals the sequential sweep in which the front heavy fills the
// next light and, on falling below A, is itself filled by the following
// heavy before any further light.  With D_i the exclusive prefix of light
// deficits (A - w) and E_j the inclusive prefix of heavy excesses (w - A):
//   light i  -> alias = heavy j* = min{j : E_j >= D_i}, threshold w_i / A;
//   heavy j with E_j < D_total -> alias = heavy j+1, kept weight
//               A - (D_i + d_i - E_j) with i the light whose deficit interval
//               [D_i, D_i + d_i) contains E_j;
//   other heavies keep the whole slot.
// Every quantity is an exact integer (K <= 32768 keeps K*A below 2^63).
// sq[K] holds q; vals[K] and idx[K] are scratch.  Block-cooperative.
// ---------------------------------------------------------------------------
__device__ void alias_build_block(const u64* sq, u32 K, u64 A, u64* vals, uint16_t* idx,
                                  u64* out_row, u64* sh) {
  const u32 NT = blockDim.x, tid = threadIdx.x;
  const u32 chunk = (K + NT - 1) / NT;
  const u32 k0 = min(K, tid * chunk), k1 = min(K, k0 + chunk);
  u64 nl = 0, dl = 0, nh = 0, eh = 0;
  for (u32 k = k0; k < k1; ++k) {
    const u64 wk = (u64)K * sq[k];
    if (wk < A) {
      ++nl;
      dl += A - wk;
    } else {
      ++nh;
      eh += wk - A;
    }
  }
  u64 nL, Dtot, nH, Etot;
  u64 ol = block_excl_scan_u64(nl, sh, &nL);
  u64 od = block_excl_scan_u64(dl, sh, &Dtot);
  u64 oh = block_excl_scan_u64(nh, sh, &nH);
  u64 oe = block_excl_scan_u64(eh, sh, &Etot);
  for (u32 k = k0; k < k1; ++k) {
    const u64 wk = (u64)K * sq[k];
    if (wk < A) {
      vals[ol] = od;
      idx[ol] = (uint16_t)k;
      od += A - wk;
      ++ol;
    } else {
      oe += wk - A;
      vals[nL + oh] = oe;
      idx[nL + oh] = (uint16_t)k;
      ++oh;
    }
  }
  __syncthreads();
  const u64* Ev = vals + nL;
  const uint16_t* Hi = idx + nL;
  for (u32 i = tid; i < (u32)nL; i += NT) {
    const u64 D = vals[i];
    u32 lo = 0, hi = (u32)nH - 1;  // first j with E_j >= D (exists: D < Dtot = E_last)
    while (lo < hi) {
      const u32 mid = (lo + hi) >> 1;
      if (Ev[mid] >= D) hi = mid; else lo = mid + 1;
    }
    const u32 l = idx[i];
    out_row[l] = ((u64)Hi[lo] << 32) | alias_threshold((u64)K * sq[l], A);
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
      const u64 d = A - (u64)K * sq[idx[lo]];
      const u64 over = vals[lo] + d - E;
      out_row[h] = ((u64)Hi[j + 1] << 32) | alias_threshold(A - over, A);
    } else {
      out_row[h] = ((u64)h << 32) | 0xffffffffu;
    }
  }
}

// Per word: q = floor(x * 2^32 / S[k]) (clamped), A, nnz, alias table.
// Persistent blocks loop over words; scratch is shared memory or, for large
// K, a per-block slice of global memory.
__global__ void __launch_bounds__(256) alias_build_kernel(ModelDev m, unsigned char* gscratch, size_t slice) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ u64 sh[33];
  const u32 K = m.K;
  unsigned char* base = gscratch ? gscratch + (size_t)blockIdx.x * slice : s_raw;
  u64* sq = (u64*)base;
  u64* vals = sq + K;
  uint16_t* idx = (uint16_t*)(vals + K);
  for (u32 w = blockIdx.x; w < m.V; w += gridDim.x) {
    const size_t row = (size_t)w * K;
    u64 part = 0, cnt = 0;
    for (u32 k = threadIdx.x; k < K; k += blockDim.x) {
      const u32 x = m.q[row + k];
      u64 qq = 0;
      if (x) {
        qq = (((u64)x) << 32) / m.S[k];
        if (qq > 0xffffffffULL) qq = 0xffffffffULL;
        ++cnt;
      }
      m.q[row + k] = (u32)qq;
      sq[k] = qq;
      part += qq;
    }
    const u64 A = block_sum_u64(part, sh);
    const u64 nz = block_sum_u64(cnt, sh);
    alias_build_block(sq, K, A, vals, idx, m.al + row, sh);
    if (threadIdx.x == 0) {
      m.A[w] = A;
      m.nnz[w] = (u32)nz;
    }
    __syncthreads();
  }
}

__global__ void debug_alias_kernel(const u32* q, u32 K, u64* out) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ u64 sh[33];
  u64* sq = (u64*)s_raw;
  u64* vals = sq + K;
  uint16_t* idx = (uint16_t*)(vals + K);
  u64 part = 0;
  for (u32 k = threadIdx.x; k < K; k += blockDim.x) {
    sq[k] = q[k];
    part += q[k];
  }
  const u64 A = block_sum_u64(part, sh);
  alias_build_block(sq, K, A, vals, idx, out, sh);
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
    d_idx[i] = (u32)off;
    off += d_len[i];
  }
}

// ---------------------------------------------------------------------------
// z sweep (reference: sample_topics, src/cu/topics.cu:36-105, with
// count_topics / compute_product_cumsum / draw_wary_search / draw_alias from
// src/cu/topics.cuh:63-192).  One warp per document; documents come from a
// global work counter.  The document's topic counts m_d live in shared memory
// as 16-bit counts plus a bitmap of nonzero topics; lane l owns bitmap words
// [l*wpl, (l+1)*wpl), i.e. a contiguous topic range, so lane order followed by
// bit order is ascending topic order.
//
// Per token (after removing its current topic):
//   B      = sum_k m_dk * q[w][k]      (u64, exact)
//   sparse iff u0 * (alpha*A[w] + B) < B
//   sparse: target = floor(u1 * B); topic = first k (ascending) whose
//           inclusive prefix of m_dk * q[w][k] exceeds target
//   dense:  slot = floor(u2 * K); topic = slot if u3 < threshold else alias
//   (alpha*A + B == 0: the topic is kept)
// then the topic is added back and n[w][topic] incremented.
// ---------------------------------------------------------------------------
struct ZKernelArgs {
  ModelDev m;
  ZLaunch z;
  u32 wpl;
  double lg_Ka;  // lgamma(K * alpha)
  double lg_a;   // lgamma(alpha)
};

__global__ void __launch_bounds__(256) z_sweep_kernel(ZKernelArgs a) {
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
    u32 nz = 0;  // distinct topics in the document
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
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      for (u32 j = 0; j < nt; ++j) {
        const u32 wj = __shfl_sync(kFullMask, my_w, j);
        const u32 zj = __shfl_sync(kFullMask, my_z, j);
        const u32 r0 = __shfl_sync(kFullMask, r.x, j);
        const u32 r1 = __shfl_sync(kFullMask, r.y, j);
        const u32 r2 = __shfl_sync(kFullMask, r.z, j);
        const u32 r3 = __shfl_sync(kFullMask, r.w, j);
        const size_t row = (size_t)wj * K;
        const u32* __restrict__ qrow = m.q + row;
        if (lane == 0) {
          const u32 c = cnt[zj] - 1u;
          cnt[zj] = (uint16_t)c;
          if (c == 0) bits[zj >> 5] &= ~(1u << (zj & 31));
        }
        __syncwarp();
        // Sparse mass over this lane's topic range, ascending.
        u64 ls = 0;
        u32 myn = 0;
        for (u32 b = 0; b < wpl; ++b) {
          const u32 wi = lane * wpl + b;
          u32 bm = bits[wi];
          myn += __popc(bm);
          while (bm) {
            const u32 k = wi * 32 + (__ffs(bm) - 1);
            bm &= bm - 1;
            ls += (u64)cnt[k] * __ldg(qrow + k);
          }
        }
        const u64 incl = warp_incl_scan_u64(ls, lane);
        const u64 B = __shfl_sync(kFullMask, incl, 31);
        const u64 Aw = __ldg(m.A + wj);
        int degenerate;
        const int sp = take_sparse(r0, m.alpha, Aw, B, &degenerate);
        u32 k;
        if (degenerate) {
          k = zj;
        } else if (sp) {
          const u64 target = scale_u32(r1, B);
          const u32 ball = __ballot_sync(kFullMask, incl > target);
          const u32 f = __ffs(ball) - 1;
          u32 kk = 0;
          if (lane == f) {
            u64 run = incl - ls;
            bool done = false;
            for (u32 b = 0; b < wpl && !done; ++b) {
              const u32 wi = lane * wpl + b;
              u32 bm = bits[wi];
              while (bm) {
                const u32 kc = wi * 32 + (__ffs(bm) - 1);
                bm &= bm - 1;
                run += (u64)cnt[kc] * __ldg(qrow + kc);
                if (run > target) {
                  kk = kc;
                  done = true;
                  break;
                }
              }
            }
          }
          k = __shfl_sync(kFullMask, kk, f);
        } else {
          const u32 s = (u32)(((u64)r2 * K) >> 32);
          const u64 e = __ldg(m.al + row + s);
          k = alias_pick(e, s, r3);
        }
        const u32 ndoc = (u32)warp_sum_u64(myn);  // nnz(m_d) without this token
        if (lane == 0) {
          const u32 c = cnt[k] + 1u;
          cnt[k] = (uint16_t)c;
          if (c == 1) bits[k >> 5] |= 1u << (k & 31);
          atomicAdd(m.n + row + k, 1u);
          const u32 nw = __ldg(m.nnz + wj);
          st_S += min(ndoc, nw);
          st_sp += (sp && !degenerate) ? 1 : 0;
          if (want_ll) {
            const u32 qk = __ldg(qrow + k);
            if (qk)
              ll_acc += log((double)qk) - 22.18070977791825;  // 32 log 2
            else
              ll_skip += 1.0;
          }
        }
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (valid) p.z[off + i] = new_z;
    }
    // distinct topics after the sweep
    u32 nz_end = 0;
    for (u32 b = 0; b < wpl; ++b) nz_end += __popc(bits[lane * wpl + b]);
    nz_end = (u32)warp_sum_u64(nz_end);
    (void)nz;
    if (lane == 0 && p.K_d) p.K_d[doc] = nz_end;
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
  const U4 r = draw4(idx[i], t, stream, 0, k0, k1);
  out[i] = poisson_draw(count[i], (double)m.beta, r, idx[i], t, stream, k0, k1, m.tables);
}

}  // namespace

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
  const u64 cells = (u64)m.K * m.V;
  const u32 blocks = (u32)std::min<u64>((cells + 255) / 256, (u64)device_sm_count() * 16);
  init_counts_kernel<<<blocks, 256, 0, s>>>(m, C);
}

void launch_phi_draw(const ModelDev& m, u32 t, cudaStream_t s) {
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

static size_t alias_smem_bytes(u32 K) { return ((size_t)K * 18 + 15) & ~(size_t)15; }

constexpr size_t kMaxDynSmem = 200 * 1024;

size_t alias_build_scratch_bytes(u32 K) {
  if (alias_smem_bytes(K) <= kMaxDynSmem) return 0;
  return alias_smem_bytes(K) * (size_t)device_sm_count() * 2;
}

void launch_alias_build(const ModelDev& m, cudaStream_t s, void* scratch, size_t scratch_bytes) {
  const u32 nt = alias_threads(m.K);
  const size_t need = alias_smem_bytes(m.K);
  if (need <= kMaxDynSmem) {
    if (need > 48 * 1024) cudaFuncSetAttribute(alias_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, alias_build_kernel, nt, need);
    if (per_sm < 1) per_sm = 1;
    const u32 blocks = std::min<u32>(m.V, (u32)(device_sm_count() * per_sm * 4));
    alias_build_kernel<<<blocks, nt, need, s>>>(m, nullptr, 0);
  } else {
    const u32 blocks = std::min<u32>(m.V, (u32)(scratch_bytes / need));
    alias_build_kernel<<<blocks, nt, 0, s>>>(m, (unsigned char*)scratch, need);
  }
}

void launch_doc_offsets(const u32* d_len, u32* d_idx, u32 n_docs, cudaStream_t s) {
  if (!n_docs) return;
  doc_offsets_kernel<<<1, 1024, 0, s>>>(d_len, d_idx, n_docs);
}

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
  a.lg_a = lgamma((double)m.alpha);
  a.lg_Ka = lgamma((double)m.K * (double)m.alpha);
  const size_t per_warp = z_sweep_smem_per_warp(m.K);
  // Warps per block: as many as fit 200 KB, at most 8.
  u32 wpb = 8;
  while (wpb > 1 && per_warp * wpb > kMaxDynSmem) --wpb;
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
  const size_t need = alias_smem_bytes(K);
  if (need > 48 * 1024) cudaFuncSetAttribute(debug_alias_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
  debug_alias_kernel<<<1, alias_threads(K), need, s>>>(q, K, out);
}

}  // namespace gpulda
