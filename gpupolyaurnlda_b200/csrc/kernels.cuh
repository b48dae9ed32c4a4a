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
  u32* nnz;    // V   nonzero x per word
  PoisTables tables;
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
  u32 flags;
  unsigned long long* counters;  // kCtrN slots, accumulated
  double* ll;                    // [0] sum, [1] skipped tokens (as double); may be null
  u32* work;                     // zeroed work-queue counter
  u32* status;
};

// Grid sizing helpers need the device's SM count.
int device_sm_count();

// n[w][k] ~ Poisson(beta + floor(C[w] / K)), iteration 0, stream kStreamInitCounts.
void launch_init_counts(const ModelDev& m, const u32* C, cudaStream_t s);
// x ~ Poisson(beta + n) into q (raw), n <- 0, S[k] += x.  S must be zeroed first.
void launch_phi_draw(const ModelDev& m, u32 t, cudaStream_t s);
// Per word: q from x and S, A, nnz and the alias table.
void launch_alias_build(const ModelDev& m, cudaStream_t s, void* scratch, size_t scratch_bytes);
size_t alias_build_scratch_bytes(u32 K);
// d_idx = exclusive scan of d_len.
void launch_doc_offsets(const u32* d_len, u32* d_idx, u32 n_docs, cudaStream_t s);
// One sweep over a set of documents.
void launch_z_sweep(const ModelDev& m, const ZLaunch& z, cudaStream_t s);
size_t z_sweep_smem_per_warp(u32 K);
// The same sweep with each document's counts in a shared-memory hash map
// (large K).  Documents longer than lmax are reported, not swept.  Returns
// false without launching when lmax needs more shared memory than a block has.
bool launch_z_sweep_map(const ModelDev& m, const ZLaunch& z, cudaStream_t s, u32 lmax);
u32 z_map_slots(u32 K, u32 lmax);

// Debug hooks.
void launch_debug_philox(const u32* ctr, u32 n, u32 k0, u32 k1, u32* out, cudaStream_t s);
void launch_debug_poisson(const ModelDev& m, const u32* count, const u64* idx, u32 n, u32 t,
                          u32 stream, u32 k0, u32 k1, u32* out, cudaStream_t s);
void launch_debug_alias(const u32* q, u32 K, u64* out, cudaStream_t s);

}  // namespace gpulda
