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
    {
      // the word's nonzero q in ascending k (thread chunks are contiguous)
      const u32 chunk = (K + blockDim.x - 1) / blockDim.x;
      const u32 k0 = min(K, threadIdx.x * chunk), k1 = min(K, k0 + chunk);
      u64 c = 0;
      for (u32 k = k0; k < k1; ++k) c += sq[k] != 0;
      u64 tot;
      u64 pos = block_excl_scan_u64(c, sh, &tot);
      for (u32 k = k0; k < k1; ++k)
        if (sq[k]) m.csr[row + pos++] = (sq[k] << 32) | k;
    }
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
