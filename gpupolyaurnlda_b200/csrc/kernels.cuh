// kernels.cuh -- launch interface of the sampler's kernels (kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace gpulda {

// Device status bits set by kernels when an input violates an invariant.
enum StatusBits : u32 {
  kStatusBadTopic = 1,    // a z value >= K (used modulo K)
  kStatusBadWord = 2,     // a w value >= V (used modulo V)
  kStatusDocRange = 4,    // a document runs past n_tokens (skipped)
  kStatusDocTooLong = 8,  // a document longer than the count width allows (skipped)
};

// Counter slots written by the z sweep.
enum CounterSlots { kCtrTokens = 0, kCtrDocs = 1, kCtrSparseWork = 2, kCtrSparseDraws = 3, kCtrN = 4 };

struct ModelDev {
  u32 K, V;
  float alpha, beta;
  u32 key0, key1;
  u32* n;      // V*K counts, word-major
  u32* q;      // V*K fixed-point Phi (raw x between the two Phi kernels)
  u64* al;     // V*K alias entries
  u64* csr;    // V*K per-word lists of (q << 32 | k) for q > 0, ascending k, nnz[w] used
  u64* A;      // V   dense mass per word
  u64* S;      // K   per-topic normalisers
  u64* Sinv;   // K   floor((2^64 - 1) / S[k]), written by the alias build's launch (null: divide)
  u32* nnz;    // V   nonzero x per word
  PoisTables tables;
};

// Problem tables of a batched launch: many independent models laid out in one
// set of arenas.  Per problem p: K, alpha, Philox key, the index of its first
// token in the concatenated corpus, lgamma(alpha), lgamma(K alpha).  Per
// global document: its problem.  Per global word: where its (word, topic) row
// starts in the arenas.
struct BatchDev {
  const u32* pid;       // per document
  const u64* row_off;   // per word
  const u32* K;
  const float* alpha;
  const u32* key0;
  const u32* key1;
  const u64* tok_base;
  const double* lg_a;
  const double* lg_Ka;
};

// Tables of the batched Phi step: per problem K, cell_base (first cell of its
// rows in the arenas), S_off (its per-topic sums), beta, Philox key, and its
// Poisson tables at offset p in the table arenas; per global word its problem
// and row offset; per block of the draw kernel (problem, first row, end row).
struct BatchPhiDev {
  const uint4* blocks;
  const u32* K;
  const u64* cell_base;
  const u64* S_off;
  const float* beta;
  const u32* key0;
  const u32* key1;
  const u32* wpid;
  const u64* row_off;
  const u32* cdf;
  const uint8_t* guide;
  const double* lfac;
};

struct ZLaunch {
  const u32* w;
  u32* z;
  const u32* d_len;
  const u32* d_idx;
  const u32* order;  // processing order of the documents (longest first); may be null
  u32* K_d;       // may be null
  u32 n_docs;
  u64 n_tokens;
  u64 tok_base;   // global index of this buffer's first token in the iteration
  u32 t;
  const u32* t_dev = nullptr;  // when set, the iteration is read from device memory (graph replays)
  u32 flags;
  unsigned long long* counters;  // kCtrN slots, accumulated
  double* ll;                    // [0] sum, [1] skipped tokens (as double); may be null
  u32* work;                     // zeroed work-queue counter
  u32* status;
};

// Grid sizing helpers need the device's SM count.
int device_sm_count();

// Host-side error reporting shared by the entry points (gpulda.cu): records
// `code` as the last error and, in fatal mode, prints and exits.
int report_error(int code, const char* what);
int report_cuda_error(cudaError_t e, const char* where);
// The single model of gpulda.h, if initialized: its device arrays and the
// iteration of its last Phi step (-1 before the first).
bool current_model(ModelDev* out, int* t);

// n[w][k] ~ Poisson(beta + floor(C[w] / K)), iteration 0, stream kStreamInitCounts.
void launch_init_counts(const ModelDev& m, const u32* C, cudaStream_t s);
void launch_init_counts_raw(u32* n, u32 K, u32 V, const u32* C, const PoisTables& tb, float beta, u32 key0, u32 key1,
                            cudaStream_t s);
// Batched Phi step: the draw over n_blocks entries of bp.blocks (the
// iteration read from t_dev; S zeroed first), then the per-word alias build
// over global words [w0, w1).  Kmax bounds the K of the problems involved.
void launch_phi_draw_batch(const ModelDev& ar, const BatchPhiDev& bp, u32 n_blocks, u32 Kmax, const u32* t_dev,
                           cudaStream_t s);
void launch_alias_build_batch(const ModelDev& ar, const BatchPhiDev& bp, u32 Kmax, u32 w0, u32 w1, cudaStream_t s);
void launch_bump(u32* t, cudaStream_t s);
// x ~ Poisson(beta + n) into q (raw), n <- 0, S[k] += x.  S must be zeroed first.
void launch_phi_draw(const ModelDev& m, u32 t, cudaStream_t s);
// Per word: q from x and S, A, nnz and the alias table.
void launch_alias_build(const ModelDev& m, cudaStream_t s, void* scratch, size_t scratch_bytes);
size_t alias_build_scratch_bytes(u32 K);
// n[w[i]][z[i]] += 1 for every token (warp-aggregated atomics); w and z
// 16-byte aligned.
void launch_count_rebuild(u32* n, const u32* w, const u32* z, u64 n_tokens, u32 K, u32 V, u32* status,
                          cudaStream_t s);
// d_idx = exclusive scan of d_len.
void launch_doc_offsets(const u32* d_len, u32* d_idx, u32 n_docs, cudaStream_t s);
// ZLaunch.flags bits.
constexpr u32 kZFlagLoglik = 1u;  // accumulate the joint log-likelihood

// One sweep over a set of documents.
void launch_z_sweep(const ModelDev& m, const ZLaunch& z, cudaStream_t s);
// One sweep over documents of many problems (arenas + tables), with the given
// warps per block and cap on blocks per SM (0: as many as fit).
void launch_z_sweep_batch(const ModelDev& arenas, const BatchDev& b, u32 Kmax, const ZLaunch& z, cudaStream_t s,
                          u32 warps_per_block, u32 blocks_per_sm);
// The same sweep with each document's counts in a shared-memory hash map
// (large K).  Documents longer than lmax are reported, not swept.  Returns
// false without launching when lmax needs more shared memory than a block has.
bool launch_z_sweep_map(const ModelDev& m, const ZLaunch& z, cudaStream_t s, u32 lmax);
u32 z_map_slots(u32 K, u32 lmax);
// The same sweep with each document's counts as a sorted list of (topic,
// count) pairs in shared memory (large K; the default there).
bool launch_z_sweep_pairs(const ModelDev& m, const ZLaunch& z, cudaStream_t s, u32 lmax);
u32 z_pairs_cap(u32 K, u32 lmax);

// Debug hooks.
void launch_debug_philox(const u32* ctr, u32 n, u32 k0, u32 k1, u32* out, cudaStream_t s);
void launch_debug_poisson(const ModelDev& m, const u32* count, const u64* idx, u32 n, u32 t,
                          u32 stream, u32 k0, u32 k1, u32* out, cudaStream_t s);
void launch_debug_alias(const u32* q, u32 K, u64* out, cudaStream_t s);

}  // namespace gpulda
