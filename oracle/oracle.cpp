// oracle.cpp -- CPU restatement of the Polya Urn LDA sweep.  TEST
// INFRASTRUCTURE ONLY: the parity tests, the smoke check and the CPU-baseline
// leg of bench.py call it as the checker; the library never links it.
//
// It restates the reference's semantics with its defects removed and shares no
// code with the CUDA library (own Philox, own tables, sequential alias
// construction, plain ascending-topic sparse walk):
//   initial counts     src/cu/polyaurn.cu:61-79   n ~ Poisson(beta + floor(C_w/K))
//   Poisson draws      src/cu/polyaurn.cu:7-36, src/cu/poisson.cu:9-20
//   Phi normalisation  src/cu/polyaurn.cu:87-123 (per-topic sums over words)
//   word-major layout  src/cu/polyaurn.cu:127-131 (transpose), 144-178 (colsums)
//   alias tables       src/cu/spalias.cu:88-174, draw src/cu/topics.cuh:63-83
//   z sweep            src/cu/topics.cu:36-105 (remove z_i, sigma_a vs sigma_b
//                      mixture, sparse inverse CDF, dense alias draw, add z_i,
//                      n[z][w] += 1), src/cu/topics.cuh:88-192
//   doc offsets        src/cu/topics.cu:5-32
//   stage order        src/cu/train.cu:137-172
// Reference defects not reproduced: the sparse term's Phi index
// (topics.cuh:174), RNG reuse across iterations (train.cu:168), overlapping RNG
// streams, unscaled alias probabilities, nondeterministic reductions.
//
// Determinism contract shared with the library: Philox4x32-10 with counter
// (index lo, index hi, iteration, stream | sub << 8) and key (seed, chain);
// integer masses; doubles only through +, -, *, /, sqrt (compiled with
// -ffp-contract=off).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

namespace {

constexpr u32 POIS_N = 64, POIS_W = 192, LFAC_N = 256, PTRS_MAX = 64;
constexpr u32 STREAM_INIT = 1, STREAM_PHI = 2, STREAM_Z = 3, STREAM_FOLD_INIT = 4, STREAM_FOLD = 5;

struct W4 {
  u32 v[4];
};

// Philox4x32-10, Salmon et al. SC'11.
W4 philox(u32 c0, u32 c1, u32 c2, u32 c3, u32 k0, u32 k1) {
  for (int r = 0; r < 10; ++r) {
    const u64 p0 = (u64)0xD2511F53u * c0;
    const u64 p1 = (u64)0xCD9E8D57u * c2;
    const u32 n0 = (u32)(p1 >> 32) ^ c1 ^ k0;
    const u32 n1 = (u32)p1;
    const u32 n2 = (u32)(p0 >> 32) ^ c3 ^ k1;
    const u32 n3 = (u32)p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return W4{{c0, c1, c2, c3}};
}

W4 draw(u64 idx, u32 t, u32 stream, u32 sub, u32 k0, u32 k1) {
  return philox((u32)idx, (u32)(idx >> 32), t, stream | (sub << 8), k0, k1);
}

double unit53(u32 a, u32 b) {
  const u64 m = ((u64)(a >> 5) << 26) | (u64)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

// log x via the atanh series on the mantissa, +,-,*,/ only.
double det_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
  u64 bits;
  std::memcpy(&bits, &x, 8);
  int e = (int)((bits >> 52) & 0x7ff) - 1023;
  const u64 mb = (bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m;
  std::memcpy(&m, &mb, 8);
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  double p = 1.0 / 23.0;
  const double inv[] = {1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0,
                        1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
  for (double c : inv) p = p * s2 + c;
  const double lm = (2.0 * s) * p;
  return (double)e * 0.6931471805599453 + lm;
}

struct Tables {
  float beta = -1.0f;
  std::vector<u32> cdf;
  std::vector<uint8_t> guide;
  std::vector<double> lfac;
};

void build_tables(float beta, Tables& T) {
  T.beta = beta;
  T.cdf.assign((size_t)POIS_N * POIS_W, 0);
  T.guide.assign((size_t)POIS_N * 256, 0);
  T.lfac.assign(LFAC_N, 0.0);
  for (u32 n = 0; n < POIS_N; ++n) {
    const double lam = (double)n + (double)beta;
    double p = std::exp(-lam), c = 0.0;
    for (u32 j = 0; j < POIS_W; ++j) {
      c += p;
      const double th = std::floor(c * 4294967296.0);
      T.cdf[n * POIS_W + j] = th >= 4294967295.0 ? 0xffffffffu : (u32)th;
      p = p * lam / (double)(j + 1);
    }
    T.cdf[n * POIS_W + POIS_W - 1] = 0xffffffffu;
    for (u32 b = 0; b < 256; ++b) {
      u32 j = 0;
      while (j < POIS_W - 1 && (u64)T.cdf[n * POIS_W + j] <= ((u64)b << 24)) ++j;
      T.guide[n * 256 + b] = (uint8_t)j;
    }
  }
  for (u32 k = 0; k < LFAC_N; ++k) T.lfac[k] = std::lgamma((double)k + 1.0);
}

double log_fact(i64 k, const Tables& T) {
  if (k < (i64)LFAC_N) return T.lfac[k];
  const double x = (double)(k + 1);
  const double ix = 1.0 / x;
  const double ix2 = ix * ix;
  double corr = ix2 * (1.0 / 1260.0) + (-1.0 / 360.0);
  corr = corr * ix2 + 1.0 / 12.0;
  corr = corr * ix;
  double r = (x + -0.5) * det_log(x);
  r = r + -x;
  r = r + 0.91893853320467274;
  return r + corr;
}

// Hoermann (1993) transformed rejection for lambda >= 10; attempt a draws the
// Philox block (idx, t, stream, sub 1 + a).
u32 ptrs(double lam, u64 idx, u32 t, u32 stream, u32 k0, u32 k1, const Tables& T) {
  const double slam = std::sqrt(lam);
  const double loglam = det_log(lam);
  const double b = 0.931 + 2.53 * slam;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b + -3.4);
  const double vr = 0.9277 + -(3.6224 / (b + -2.0));
  for (u32 att = 0; att < PTRS_MAX; ++att) {
    const W4 r = draw(idx, t, stream, 1 + att, k0, k1);
    const double U = unit53(r.v[0], r.v[1]) + -0.5;
    const double V = unit53(r.v[2], r.v[3]);
    const double us = 0.5 + -std::fabs(U);
    const double kf = std::floor(((2.0 * a) / us + b) * U + lam + 0.43);
    if (us >= 0.07 && V <= vr) return (u32)kf;
    if (kf < 0.0 || (us < 0.013 && V > us)) continue;
    const i64 k = (i64)kf;
    const double lhs = det_log((V * inv_alpha) / (a / (us * us) + b));
    const double rhs = (-lam + kf * loglam) + -log_fact(k, T);
    if (lhs <= rhs) return (u32)k;
  }
  return (u32)std::floor(lam);
}

// Cell idx's inversion word: word (idx & 3) of the Philox block (idx >> 2, t,
// stream, sub 0) -- four cells share one block.
u32 cell_word(u64 idx, u32 t, u32 stream, u32 k0, u32 k1) {
  return draw(idx >> 2, t, stream, 0, k0, k1).v[idx & 3];
}

u32 poisson(u32 n, float beta, u64 idx, u32 t, u32 stream, u32 k0, u32 k1, const Tables& T) {
  if (n < POIS_N) {
    const u32 u = cell_word(idx, t, stream, k0, k1);
    const u32* row = &T.cdf[(size_t)n * POIS_W];
    u32 j = 0;  // plain linear inversion (the guide is only a shortcut)
    while (j < POIS_W - 1 && u >= row[j]) ++j;
    return j;
  }
  return ptrs((double)n + (double)beta, idx, t, stream, k0, k1, T);
}

Tables& tables_for(float beta) {
  static thread_local Tables T;
  if (T.beta != beta) build_tables(beta, T);
  return T;
}

u32 threshold(u64 p, u64 A) {
  if (A == 0 || p >= A) return 0xffffffffu;
  const double t = std::floor(((double)p * 4294967296.0) / (double)A);
  return t >= 4294967295.0 ? 0xffffffffu : (u32)t;
}

// Sequential alias sweep over n items with integer weights q (Vose's method
// with the heavy that falls below the slot capacity filled next).  Entry of
// item i: threshold | key[i] << 32 | key[alias item] << 48.
void alias_seq(const u64* q, const uint16_t* key, u32 K, u64* out) {
  u64 A = 0;
  for (u32 k = 0; k < K; ++k) A += q[k];
  std::vector<u64> w(K);
  std::vector<u32> L, H;
  for (u32 k = 0; k < K; ++k) {
    w[k] = (u64)K * q[k];
    (w[k] < A ? L : H).push_back(k);
  }
  auto entry = [&](u32 item, u32 alias_item, u32 thr) {
    return ((u64)key[alias_item] << 48) | ((u64)key[item] << 32) | thr;
  };
  size_t li = 0, hj = 0;
  long pending = -1;
  while (true) {
    u32 l;
    if (pending >= 0) {
      l = (u32)pending;
      pending = -1;
    } else if (li < L.size()) {
      l = L[li++];
    } else {
      break;
    }
    if (hj >= H.size()) {  // unreachable with exact integer weights
      out[l] = entry(l, l, 0xffffffffu);
      continue;
    }
    const u32 h = H[hj];
    out[l] = entry(l, h, threshold(w[l], A));
    w[h] -= A - w[l];
    if (w[h] < A) {
      pending = h;
      ++hj;
    }
  }
  for (; hj < H.size(); ++hj) out[H[hj]] = entry(H[hj], H[hj], 0xffffffffu);
}

template <class F>
void parallel_for(u64 n, int threads, F f) {
  if (threads <= 1 || n < 2) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> ts;
  const u64 chunk = (n + threads - 1) / threads;
  for (int i = 0; i < threads; ++i) {
    const u64 a = std::min<u64>(n, i * chunk), b = std::min<u64>(n, a + chunk);
    if (a >= b) break;
    ts.emplace_back(f, a, b, i);
  }
  for (auto& t : ts) t.join();
}

}  // namespace

extern "C" {
u32 orc_alias_draw(const u64* table, u32 n, u32 r_slot, u32 r_keep);

void orc_philox(const u32* ctr, u32 n, u32 k0, u32 k1, u32* out) {
  for (u32 i = 0; i < n; ++i) {
    const W4 r = philox(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], k0, k1);
    for (int j = 0; j < 4; ++j) out[4 * i + j] = r.v[j];
  }
}

void orc_tables(float beta, u32* cdf, uint8_t* guide, double* lfac) {
  Tables T;
  build_tables(beta, T);
  if (cdf) std::memcpy(cdf, T.cdf.data(), T.cdf.size() * 4);
  if (guide) std::memcpy(guide, T.guide.data(), T.guide.size());
  if (lfac) std::memcpy(lfac, T.lfac.data(), T.lfac.size() * 8);
}

void orc_poisson(const u32* count, const u64* idx, u32 n, float beta, u32 t, u32 stream, u32 k0, u32 k1, u32* out) {
  const Tables& T = tables_for(beta);
  for (u32 i = 0; i < n; ++i) out[i] = poisson(count[i], beta, idx[i], t, stream, k0, k1, T);
}

double orc_log(double x) { return det_log(x); }

// n[w*K+k] ~ Poisson(beta + floor(C[w] / K)) with stream 1, iteration 0.
void orc_init_counts(u32 K, u32 V, float beta, const u32* C, u32 k0, u32 k1, u32* n, int threads) {
  parallel_for(V, threads, [&](u64 a, u64 b, int) {
    const Tables& T = tables_for(beta);
    for (u64 w = a; w < b; ++w)
      for (u32 k = 0; k < K; ++k) {
        const u64 c = w * K + k;
        n[c] = poisson(C[w] / K, beta, c, 0, STREAM_INIT, k0, k1, T);
      }
  });
}

// Phi step of iteration t from counts n (word-major, unchanged):
// x = Poisson(beta + n); S[k] = sum_w x; q = floor(x 2^32 / S[k]) clamped;
// A[w] = sum_k q; nnz[w] = #{k: x > 0}; alias tables.
void orc_phi_step(u32 K, u32 V, float beta, const u32* n, u32 t, u32 k0, u32 k1, u32* q, u64* al, u64* A, u64* S,
                  u32* nnz, int threads) {
  const int nt = std::max(1, threads);
  std::vector<std::vector<u64>> part(nt, std::vector<u64>(K, 0));
  parallel_for(V, nt, [&](u64 a, u64 b, int tid) {
    const Tables& T = tables_for(beta);
    std::vector<u64>& ps = part[tid];
    for (u64 w = a; w < b; ++w)
      for (u32 k = 0; k < K; ++k) {
        const u64 c = w * K + k;
        const u32 x = poisson(n[c], beta, c, t, STREAM_PHI, k0, k1, T);
        q[c] = x;
        ps[k] += x;
      }
  });
  for (u32 k = 0; k < K; ++k) {
    u64 s = 0;
    for (int i = 0; i < nt; ++i) s += part[i][k];
    S[k] = s;
  }
  // per word: the topics with q > 0 in ascending order carry the word's
  // sparse alias table (entries 0 .. nnz-1 of the row; the rest unused)
  parallel_for(V, nt, [&](u64 a, u64 b, int) {
    std::vector<u64> row;
    std::vector<uint16_t> keys;
    for (u64 w = a; w < b; ++w) {
      u64 sum = 0;
      row.clear();
      keys.clear();
      for (u32 k = 0; k < K; ++k) {
        const u64 c = w * K + k;
        const u32 x = q[c];
        u64 v = 0;
        if (x) {
          v = ((u64)x << 32) / S[k];
          if (v > 0xffffffffULL) v = 0xffffffffULL;
        }
        q[c] = (u32)v;
        if (v) {
          row.push_back(v);
          keys.push_back((uint16_t)k);
        }
        sum += v;
      }
      A[w] = sum;
      nnz[w] = (u32)row.size();
      std::fill(al + w * K, al + w * K + K, 0ull);
      if (!row.empty()) alias_seq(row.data(), keys.data(), (u32)row.size(), al + w * K);
    }
  });
}

// Alias table over K items with topics 0..K-1.
void orc_alias(const u32* q, u32 K, u64* out) {
  std::vector<u64> row(q, q + K);
  std::vector<uint16_t> keys(K);
  for (u32 k = 0; k < K; ++k) keys[k] = (uint16_t)k;
  alias_seq(row.data(), keys.data(), K, out);
}

// Alias table over n items with the given topics.
void orc_alias_items(const u32* q, const uint16_t* keys, u32 n, u64* out) {
  std::vector<u64> row(q, q + n);
  alias_seq(row.data(), keys, n, out);
}

// Dense draw (reference draw_alias, src/cu/topics.cuh:63-83) from a table of
// n slots: slot = floor(r_slot * n / 2^32); the slot's own topic when
// r_keep < threshold, else its alias topic.
u32 orc_alias_draw(const u64* table, u32 n, u32 r_slot, u32 r_keep) {
  const u32 slot = (u32)(((u64)r_slot * n) >> 32);
  const u64 e = table[slot];
  return r_keep < (u32)e ? (u32)(e >> 32) & 0xffffu : (u32)(e >> 48);
}

// Sparse inverse CDF (reference draw_wary_search over the prefix of
// compute_product_cumsum, src/cu/topics.cuh:88-192): masses in the given order;
// target = floor(r * total / 2^32); returns the first index whose inclusive
// prefix exceeds the target, and writes the inclusive prefix.
u32 orc_sparse_select(const u64* mass, u32 n, u32 r, u64* prefix) {
  u64 B = 0;
  for (u32 i = 0; i < n; ++i) {
    B += mass[i];
    if (prefix) prefix[i] = B;
  }
  const u64 target = (u64)r * (B >> 32) + (((u64)r * (B & 0xffffffffULL)) >> 32);
  u64 run = 0;
  for (u32 i = 0; i < n; ++i) {
    run += mass[i];
    if (run > target) return i;
  }
  return n;
}

// Topic counts of one document (reference count_topics, src/cu/topics.cuh:142-158).
u32 orc_count_topics(const u32* z, u32 L, u32 K, u32* counts) {
  std::fill(counts, counts + K, 0u);
  u32 distinct = 0;
  for (u32 i = 0; i < L; ++i)
    if (counts[z[i] % K]++ == 0) ++distinct;
  return distinct;
}

// Exclusive scan of document lengths.
void orc_doc_offsets(const u32* d_len, u32 n_docs, u64* d_idx) {
  u64 s = 0;
  for (u32 i = 0; i < n_docs; ++i) {
    d_idx[i] = s;
    s += d_len[i];
  }
}

// New topic of a token whose current topic zi has already been removed from
// the document's counts m (nonzero topics flagged in bits): the mixture of
// the sparse part sum_k m_k q[k] and the dense part alpha * A (src/cu/
// topics.cu:36-105, topics.cuh:63-192).  *sparse: the sparse part chose it.
static u32 draw_topic(u32 K, float alpha, const u32* qrow, const u64* alrow, u64 Aw, u32 nnzw, const u32* m,
                      const u64* bits, u32 nwords, const W4& r, u32 zi, bool* sparse) {
  u64 B = 0;
  for (u32 bw = 0; bw < nwords; ++bw)
    for (u64 bm = bits[bw]; bm; bm &= bm - 1) {
      const u32 k = bw * 64 + (u32)__builtin_ctzll(bm);
      B += (u64)m[k] * qrow[k];
    }
  const double tot = (double)alpha * (double)Aw + (double)B;
  const double u = (double)r.v[0] * (1.0 / 4294967296.0);
  *sparse = false;
  if (!(tot > 0.0)) return zi;
  if (u * tot < (double)B) {
    *sparse = true;
    const u64 target = (u64)r.v[1] * (B >> 32) + (((u64)r.v[1] * (B & 0xffffffffULL)) >> 32);
    u64 run = 0;
    for (u32 bw = 0; bw < nwords; ++bw)
      for (u64 bm = bits[bw]; bm; bm &= bm - 1) {
        const u32 kc = bw * 64 + (u32)__builtin_ctzll(bm);
        run += (u64)m[kc] * qrow[kc];
        if (run > target) return kc;
      }
    return K;  // unreachable: the prefix reaches B > target
  }
  // dense part: the word's sparse alias table has nnzw slots
  return orc_alias_draw(alrow, nnzw, r.v[2], r.v[3]);
}

// One z sweep over n_docs documents laid out back to back in w/z.
// n_out (word-major, V*K) is incremented for every token's new topic.
// stats[0] += tokens, [1] += docs, [2] += sum min(nnz(m_d^-i), nnz[w]),
// [3] += sparse draws.  ll[0] += joint log-likelihood terms, ll[1] += tokens
// with q = 0.  K_d_out (optional) receives distinct topics per document.
void orc_z_sweep(u32 K, u32 V, float alpha, const u32* q, const u64* al, const u64* A, const u32* nnz, const u32* w,
                 u32* z, const u32* d_len, u32 n_docs, u64 tok_base, u32 t, u32 k0, u32 k1, u32* n_out, u64* stats,
                 double* ll, u32* K_d_out, int threads) {
  std::vector<u64> offs(n_docs);
  orc_doc_offsets(d_len, n_docs, offs.data());
  const int nt = std::max(1, threads);
  std::vector<u64> st(4 * nt, 0);
  std::vector<double> lls(2 * nt, 0.0);
  const double lg_a = std::lgamma((double)alpha);
  const double lg_Ka = std::lgamma((double)K * (double)alpha);
  const u32 nwords = (K + 63) / 64;
  parallel_for(n_docs, nt, [&](u64 a, u64 b, int tid) {
    std::vector<u32> m(K, 0);
    std::vector<u64> bits(nwords, 0);
    u64 s_tok = 0, s_S = 0, s_sp = 0;
    double s_ll = 0.0, s_skip = 0.0;
    for (u64 d = a; d < b; ++d) {
      const u64 off = offs[d];
      const u32 L = d_len[d];
      std::fill(m.begin(), m.end(), 0);
      std::fill(bits.begin(), bits.end(), 0);
      u32 nzd = 0;
      for (u32 i = 0; i < L; ++i) {
        const u32 k = z[off + i] % K;
        if (m[k]++ == 0) {
          bits[k >> 6] |= 1ull << (k & 63);
          ++nzd;
        }
      }
      for (u32 i = 0; i < L; ++i) {
        const u32 wi = w[off + i] % V;
        const u32 zi = z[off + i] % K;
        const u64 row = (u64)wi * K;
        if (--m[zi] == 0) {
          bits[zi >> 6] &= ~(1ull << (zi & 63));
          --nzd;
        }
        const W4 r = draw(tok_base + off + i, t, STREAM_Z, 0, k0, k1);
        bool sparse = false;
        const u32 k = draw_topic(K, alpha, q + row, al + row, A[wi], nnz[wi], m.data(), bits.data(), nwords, r, zi,
                                 &sparse);
        s_S += std::min<u64>(nzd, nnz[wi]);
        s_sp += sparse ? 1 : 0;
        if (m[k]++ == 0) {
          bits[k >> 6] |= 1ull << (k & 63);
          ++nzd;
        }
        __atomic_fetch_add(&n_out[row + k], 1u, __ATOMIC_RELAXED);
        z[off + i] = k;
        if (ll) {
          const u32 qk = q[row + k];
          if (qk)
            s_ll += std::log((double)qk) - 22.18070977791825;
          else
            s_skip += 1.0;
        }
      }
      if (ll) {
        double dl = 0.0;
        for (u32 bw = 0; bw < nwords; ++bw)
          for (u64 bm = bits[bw]; bm; bm &= bm - 1) {
            const u32 kc = bw * 64 + (u32)__builtin_ctzll(bm);
            dl += std::lgamma((double)alpha + (double)m[kc]) - lg_a;
          }
        s_ll += dl + lg_Ka - std::lgamma((double)K * (double)alpha + (double)L);
      }
      if (K_d_out) K_d_out[d] = nzd;
      s_tok += L;
    }
    st[4 * tid + 0] = s_tok;
    st[4 * tid + 1] = b - a;
    st[4 * tid + 2] = s_S;
    st[4 * tid + 3] = s_sp;
    lls[2 * tid] = s_ll;
    lls[2 * tid + 1] = s_skip;
  });
  if (stats)
    for (int i = 0; i < nt; ++i)
      for (int j = 0; j < 4; ++j) stats[j] += st[4 * i + j];
  if (ll)
    for (int i = 0; i < nt; ++i) {
      ll[0] += lls[2 * i];
      ll[1] += lls[2 * i + 1];
    }
}

// Fold-in of new documents against a fixed model (no count rebuild).  For
// document r (length len[r], id ids[r]): topics start at floor(u * K) with
// u from Philox (token, id low bits, 0, STREAM_FOLD_INIT) under key (k0,
// k1 ^ id high bits), then n_iter sweeps draw every token as the z sweep does
// with counter (token, id low bits, iteration, STREAM_FOLD).  Outputs
// theta[r][k] = (float)((m_k + alpha) / (L + K alpha)), the log-likelihood
// sum_i log sum_k theta_k q[w_i][k] / 2^32 over tokens whose word has mass
// (the others are counted in skipped), and the final topics in z_out.
void orc_fold_in(u32 K, u32 V, float alpha, const u32* q, const u64* al, const u64* A, const u32* nnz, const u32* w,
                 const u32* len, const u64* ids, u32 n_docs, u32 k0, u32 k1, u32 n_iter, float* theta, double* ll,
                 u32* skipped, u32* z_out, int threads) {
  std::vector<u64> offs(n_docs);
  orc_doc_offsets(len, n_docs, offs.data());
  const u32 nwords = (K + 63) / 64;
  parallel_for(n_docs, std::max(1, threads), [&](u64 a, u64 b, int) {
    std::vector<u32> m(K);
    std::vector<u64> bits(nwords);
    for (u64 d = a; d < b; ++d) {
      const u32 L = len[d];
      const u32* wd = w + offs[d];
      u32* z = z_out + offs[d];
      const u64 ridx = (u64)(u32)ids[d] << 32;
      const u32 kk1 = k1 ^ (u32)(ids[d] >> 32);
      std::fill(m.begin(), m.end(), 0);
      std::fill(bits.begin(), bits.end(), 0);
      for (u32 i = 0; i < L; ++i) {
        const W4 r = draw(ridx | i, 0, STREAM_FOLD_INIT, 0, k0, kk1);
        z[i] = (u32)(((u64)r.v[0] * K) >> 32);
        if (m[z[i]]++ == 0) bits[z[i] >> 6] |= 1ull << (z[i] & 63);
      }
      for (u32 t = 0; t < n_iter; ++t)
        for (u32 i = 0; i < L; ++i) {
          const u32 wi = wd[i] % V, zi = z[i];
          const u64 row = (u64)wi * K;
          if (--m[zi] == 0) bits[zi >> 6] &= ~(1ull << (zi & 63));
          const W4 r = draw(ridx | i, t, STREAM_FOLD, 0, k0, kk1);
          bool sparse;
          const u32 k = draw_topic(K, alpha, q + row, al + row, A[wi], nnz[wi], m.data(), bits.data(), nwords, r,
                                   zi, &sparse);
          if (m[k]++ == 0) bits[k >> 6] |= 1ull << (k & 63);
          z[i] = k;
        }
      const double denom = (double)L + (double)K * (double)alpha;
      for (u32 k = 0; k < K; ++k) theta[d * K + k] = (float)(((double)m[k] + (double)alpha) / denom);
      double s_ll = 0.0;
      u32 skip = 0;
      for (u32 i = 0; i < L; ++i) {
        const u64 row = (u64)(wd[i] % V) * K;
        double s = 0.0;
        for (u32 k = 0; k < K; ++k)
          if (q[row + k]) s += ((double)m[k] + (double)alpha) * (double)q[row + k];
        if (s > 0.0)
          s_ll += std::log(s);
        else
          ++skip;
      }
      ll[d] = s_ll - (double)(L - skip) * (std::log(denom) + 22.18070977791825);
      skipped[d] = skip;
    }
  });
}

}  // extern "C"
