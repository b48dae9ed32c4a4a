/*
 * gpulda.h -- C ABI of libGPUPolyaUrnLDA.so, the B200 (sm_100a) Polya Urn LDA
 * Gibbs sampler.
 *
 * The first five entry points and the two structs are the reference's ABI,
 * bound by its Rust host (src/ffi.rs:4-31, src/buffer.rs:4-19) and declared by
 * its CUDA side in src/cu/train.cuh:13-45.  Layouts and symbol names are
 * identical, so the reference's train.rs drives this library unchanged.
 *
 * Everything prefixed gpulda_ is an addition: seeds, a non-exiting error mode,
 * log-likelihood, per-kernel timings, a device-resident corpus mode used for
 * benchmarking, and read-back hooks used by the parity tests.
 *
 * Semantics (shared by every entry point):
 *   - one model per process; calls come from one host thread;
 *   - iteration t = number of sample_phi() calls made so far minus one;
 *   - random numbers are Philox4x32-10 keyed by (seed, chain) with counter
 *     (index, t, stream), so results do not depend on launch shapes or on how
 *     the corpus is split into buffers;
 *   - counts are exact integers; Phi is held as 32-bit fixed point
 *     q[w][k] = floor(x[k][w] * 2^32 / S[k]) (clamped to 2^32-1), where
 *     x ~ Poisson(beta + n[k][w]) and S[k] = sum_w x[k][w].
 */
#ifndef GPULDA_H
#define GPULDA_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Model arguments.  Same layout as Args in src/cu/train.cuh:13-21 and
 * Args_FFI in src/ffi.rs:4-13 (32 bytes on x86-64, C at offset 16).
 * C holds V word counts (word ids ranked by descending count, as
 * src/preprocess.rs:23-28 writes them).  The library copies what it needs
 * during initialize and does not keep the pointer. */
typedef struct Args {
  float alpha;
  float beta;
  uint32_t K;
  uint32_t V;
  uint32_t* C;
  uint32_t buffer_size; /* max tokens per buffer */
  uint32_t max_D;       /* max documents per buffer */
} Args;

/* One streaming buffer.  Same layout as Buffer in src/cu/train.cuh:23-37 and
 * src/buffer.rs:4-19 (96 bytes on x86-64).  z, w, d (document lengths) and
 * K_d are host arrays owned by the caller; z must be writable, w/d/K_d may be
 * read-only mappings (the library never writes them).  The seven gpu_* /
 * stream slots are owned by the library: filled by initialize, released by
 * cleanup.  gpu_rng holds the library's per-buffer context (the counter-based
 * generator keeps no state); stream holds a cudaStream_t*. */
typedef struct Buffer {
  uint32_t* z;
  uint32_t* w;
  uint32_t* d;
  uint32_t* K_d;
  uint32_t n_docs;
  uint32_t n_tokens;
  void* gpu_z;
  void* gpu_w;
  void* gpu_d_len;
  void* gpu_d_idx;
  void* gpu_K_d;
  void* gpu_rng;
  void* stream;
} Buffer;

/* ---- reference ABI (src/cu/train.cuh:41-45, src/ffi.rs:16-31) ---------- */

/* Replaces initialize() (src/cu/train.cu:31-96): allocates the model, the
 * n_buffers buffers' device storage and streams, and draws the initial
 * counts n[k][w] ~ Poisson(beta + floor(C[w] / K)) (src/cu/polyaurn.cu:61-79).
 * Seed 0, chain 0. */
void initialize(Args* args, Buffer* buffers, uint32_t n_buffers);

/* Replaces sample_phi() (src/cu/train.cu:137-156): draws x ~ Poisson(beta+n),
 * the per-topic normalisers S, the fixed-point Phi q, the per-word dense mass
 * A[w] = sum_k q[w][k] and the per-word alias tables; then zeroes n so the
 * following sweep rebuilds it.  Synchronous, like the reference. */
void sample_phi(void);

/* Replaces sample_z_async() (src/cu/train.cu:158-172): copies the buffer's
 * z, w, d, K_d to the device, computes document offsets, resamples every
 * token's topic and rebuilds n, then copies z back.  Returns before the work
 * completes. */
void sample_z_async(Buffer* buffer);

/* Buffers are independent on the device (own arrays, streams and work
 * counters): a host may keep several in flight, calling sample_z_async on the
 * next buffer before sync_buffer on the previous one (token numbering follows
 * the order of the sample_z_async calls).  Every buffer must be synced before
 * the next sample_phi. */

/* Replaces sync_buffer() (src/cu/train.cu:174-177): waits for the buffer. */
void sync_buffer(Buffer* buffer);

/* Replaces cleanup() (src/cu/train.cu:98-135): frees everything. */
void cleanup(Buffer* buffers, uint32_t n_buffers);

/* ---- additions ---------------------------------------------------------- */

/* Error codes.  The five legacy entry points return void: by default an error
 * prints a message and exits the process (the reference's behaviour,
 * src/cu/error.cuh:13-18).  gpulda_set_fatal_errors(0) makes them record the
 * error instead; gpulda_last_error() returns and clears it. */
enum {
  GPULDA_OK = 0,
  GPULDA_ERR_CUDA = 1,        /* a CUDA runtime call failed */
  GPULDA_ERR_ARGS = 2,        /* invalid model arguments */
  GPULDA_ERR_STATE = 3,       /* call out of protocol order */
  GPULDA_ERR_BUFFER = 4,      /* buffer exceeds buffer_size / max_D, or bad doc */
  GPULDA_ERR_NOMEM = 5,       /* device allocation failed */
  GPULDA_ERR_DEVICE = 6,      /* a kernel reported a violated invariant */
  GPULDA_ERR_UNSUPPORTED = 7  /* size outside what this build supports */
};
int gpulda_last_error(void);
const char* gpulda_error_string(int code);
void gpulda_set_fatal_errors(int fatal);

/* Limits of this build. */
#define GPULDA_MAX_K 32768u          /* topics (16-bit topic ids on device) */
#define GPULDA_MAX_DOC_LEN 65535u    /* tokens per document (16-bit counts) */

typedef struct GpuldaExArgs {
  uint64_t seed;   /* Philox key word 0 (low 32 bits used) */
  uint32_t chain;  /* Philox key word 1: independent chains / replicas */
  uint32_t flags;  /* GPULDA_FLAG_* */
} GpuldaExArgs;

#define GPULDA_FLAG_LOGLIK 1u  /* accumulate the joint log-likelihood per sweep */
/* K > 2048: keep each document's counts in the order-preserving Robin Hood
 * hash map instead of the default sorted (topic, count) list (same results). */
#define GPULDA_FLAG_HASHMAP 2u

/* initialize() with an explicit seed, chain id and flags. Returns an error
 * code (never exits). */
int gpulda_initialize_ex(const Args* args, Buffer* buffers, uint32_t n_buffers,
                         const GpuldaExArgs* ex);

/* Runs all library work on the given cudaStream_t (0 restores the library's
 * own streams).  Lets a caller time the library with its own CUDA events. */
int gpulda_set_stream(void* cuda_stream);

/* Joint log-likelihood of the last completed iteration (all buffers swept
 * since the last sample_phi), using the Phi that sweep used:
 *   sum_i log Phi[z_i][w_i]
 * + sum_d [lgamma(K a) - lgamma(K a + L_d)
 *          + sum_{k: m_dk>0} (lgamma(a + m_dk) - lgamma(a))].
 * Needs GPULDA_FLAG_LOGLIK.  n_skipped (optional) receives the number of
 * tokens whose Phi was zero (left out of the first sum). */
int gpulda_loglik(double* out, uint64_t* n_skipped);

/* Device-resident corpus (no host copies per iteration).  Load copies the
 * corpus to the device once; sweep runs n_iter full iterations
 * (sample_phi + one z sweep over the whole corpus); read_z copies z back. */
int gpulda_corpus_load(const uint32_t* z, const uint32_t* w, const uint32_t* d_len,
                       uint32_t n_docs, uint64_t n_tokens);
int gpulda_corpus_sweep(uint32_t n_iter);
int gpulda_corpus_read_z(uint32_t* z_out);
/* Rebuilds the count table n from the resident corpus's current topics
 * (n[w][z] = tokens of word w with topic z; warp-aggregated atomics), e.g. to
 * resume a chain from saved topics instead of the initial counts of
 * initialize.  The next sample_phi draws Phi from these counts.  ms
 * (optional) receives the rebuild kernel's device time.  No counterpart in
 * the reference, whose rebuild is the per-token atomicAdd of sample_topics
 * (src/cu/topics.cu:95); the sweeps here rebuild n the same way as they go. */
int gpulda_corpus_count_rebuild(float* ms);

/* Per-kernel device times (ms) of the last iteration, in this order:
 * [0] Phi/Poisson draw, [1] normaliser prep, [2] alias build,
 * [3] document offsets, [4] z sweep (+count rebuild).  Returns the number of
 * entries written (<= n). */
int gpulda_kernel_times(float* ms, int n);

/* Counters of the last iteration: [0] tokens swept, [1] documents,
 * [2] sparse work S = sum over tokens of min(nnz(m_d without the token),
 * nnz(x[.][w])), [3] tokens that took the sparse branch,
 * [4] kernels launched by the library in that iteration. */
int gpulda_counters(uint64_t* out, int n);

/* Document sharding across processes, one GPU each.  Every process holds the
 * whole model (same arguments, seed and chain) and sweeps only its own range
 * of documents.  gpulda_set_token_offset gives the global index, in the whole
 * corpus, of the process's first token: the numbering of the next buffer and
 * of every later iteration (after each sample_phi) starts there, so each token
 * gets the draws the single-process chain gives it.  After its sweeps, the
 * processes add their count tables in place (gpulda_count_table: the device
 * array n, K*V uint32, e.g. an all-reduce sum over NCCL) before any of them
 * calls sample_phi again; every process then computes the same Phi, and the
 * chain equals the single-process chain bit for bit.  Log-likelihoods add
 * likewise (gpulda_loglik returns the process's part). */
int gpulda_set_token_offset(uint64_t first_token);
int gpulda_count_table(void** device_ptr, uint64_t* n_cells);

/* Page-locks (pins) a host range so the copies of sample_z_async / sync_buffer
 * from and to it run as asynchronous DMA; e.g. the memory-mapped z/w/d/K_d
 * files of a streaming host loop.  GPULDA_PIN_READ_ONLY for ranges mapped
 * read-only.  Unpin before unmapping.  Returns GPULDA_ERR_CUDA if the range
 * cannot be pinned (the copies then still work, staged by the driver). */
#define GPULDA_PIN_READ_ONLY 1u
int gpulda_pin_host(void* p, uint64_t bytes, uint32_t flags);
int gpulda_unpin_host(void* p);

/* ---- read-back hooks for the parity tests ------------------------------ */

/* Copies model state to host arrays (any pointer may be NULL):
 * n      V*K uint32  counts, word-major n[w*K+k]
 * q      V*K uint32  fixed-point Phi, word-major
 * alias  V*K uint64  alias tables: low 32 bits threshold, high 32 bits alias
 * A      V   uint64  per-word dense mass sum_k q[w][k]
 * S      K   uint64  per-topic normalisers sum_w x[k][w]
 * nnz    V   uint32  number of k with x[k][w] > 0 */
int gpulda_debug_read(uint32_t* n, uint32_t* q, uint64_t* alias, uint64_t* A,
                      uint64_t* S, uint32_t* nnz);
/* Overwrites the counts n (V*K uint32, word-major). */
int gpulda_debug_write_counts(const uint32_t* n);
/* Copies the Poisson inversion tables built at initialize:
 * cdf  GPULDA_POIS_TABLE_N * GPULDA_POIS_TABLE_W uint32 thresholds,
 * lfac GPULDA_LOGFAC_N doubles (log k!). */
#define GPULDA_POIS_TABLE_N 64u
#define GPULDA_POIS_TABLE_W 192u
#define GPULDA_LOGFAC_N 256u
int gpulda_debug_tables(uint32_t* cdf, double* lfac);

/* Runs the device Philox4x32-10 on n counters (4 words each) with one key;
 * writes 4 words per counter.  Used to pin the device generator against
 * published known-answer vectors. */
int gpulda_debug_philox(const uint32_t* ctr, uint32_t n, uint32_t key0, uint32_t key1,
                        uint32_t* out);

/* Runs the device Poisson sampler for n (count, counter) pairs:
 * out[i] = Poisson(beta + count[i]) drawn with counter
 * (idx[i], t, stream) under (key0, key1).  Requires an initialized model
 * (the tables depend on beta). */
int gpulda_debug_poisson(const uint32_t* count, const uint64_t* idx, uint32_t n,
                         uint32_t t, uint32_t stream, uint32_t key0, uint32_t key1,
                         uint32_t* out);

/* Builds one alias table on the device from integer weights q[0..K) with
 * the library's parallel construction; writes K packed entries. */
int gpulda_debug_alias(const uint32_t* q, uint32_t K, uint64_t* table_out);

/* ---- allocation-free sweep ------------------------------------------------
 * No counterpart in the reference: an addition for callers that must not
 * allocate device memory when they call (a host application that owns all
 * device memory through its own pool, a service that allocates nothing once
 * it is serving, or work issued where cudaMalloc is not permitted).
 *
 * Sweeps n_docs documents whose topics z (read and rewritten), words w and
 * lengths d_len are already in device memory with the draws and count rebuild
 * of sample_z_async, continuing the current iteration's token numbering (for
 * K above 2048 with the large-K store sized for K distinct topics per
 * document).  Asynchronous on `stream` (NULL: the library's stream); device-side
 * input errors are reported by the next sync_buffer / sample_phi /
 * gpulda_corpus_* call.  Per-document distinct-topic counts (K_d) are not
 * written and gpulda_kernel_times does not cover this call.
 *
 * Ordering: the next sample_phi (and gpulda_corpus_sweep) waits on the GPU
 * for the last allocation-free sweep, whatever stream it ran on, so the caller
 * need not synchronize its stream before sample_phi; gpulda_loglik,
 * gpulda_counters and gpulda_debug_read synchronize the device.  Calls made
 * one after another from the host are ordered on the GPU as well.
 *
 * It allocates nothing: its scratch (document offsets and a work counter) is
 * a fixed device array of the library, 4 MiB + 256 B held by every GPU that
 * loads the library until the process exits.  n_docs above
 * GPULDA_NOALLOC_MAX_DOCS is rejected with GPULDA_ERR_UNSUPPORTED.  The first
 * call on a device looks up that array's address, so make the first call
 * before any stream capture.  Calls share the array: calls whose work
 * overlaps on the GPU (issued from several host threads, say) race with each
 * other. */
#define GPULDA_NOALLOC_MAX_DOCS 1048576u
int gpulda_sample_z_device_noalloc(uint32_t* z, const uint32_t* w, const uint32_t* d_len, uint32_t n_docs,
                                   uint64_t n_tokens, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GPULDA_H */
