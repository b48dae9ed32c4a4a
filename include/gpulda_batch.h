/*
 * gpulda_batch.h -- batched chains: many independent LDA problems swept
 * together on one GPU (exported by libGPUPolyaUrnLDA.so).
 *
 * No counterpart in the reference, whose ABI (src/cu/train.cuh:41-45) holds
 * one model per process.  Each problem here is exactly what one
 * gpulda_initialize_ex + gpulda_corpus_load + gpulda_corpus_sweep(n) run of
 * include/gpulda.h computes for the same arguments, seed and chain: the same
 * Philox counters (problem-local cell and token indices), so every problem's
 * topics and counts equal its solo run bit for bit, and its log-likelihood
 * equals the solo value up to the order of floating-point sums.
 *
 * Layout: all problems' (word, topic) rows, word vectors, per-topic sums,
 * tokens and documents live in shared device arenas, grouped by K bucket
 * (K <= 64, <= 256, <= 1024, <= 2048).  One iteration of every problem is
 * one CUDA graph, the iteration number read from device memory so the same
 * graph replays for every iteration.  In the merged mode the graph holds one
 * launch per stage for all problems: a Poisson draw over every problem's
 * rows, an alias build over every word, and one persistent z sweep whose
 * warps take (problem, document) items, longest first, from a single work
 * queue spanning all buckets.  In the merged-sweep mode (the default) each
 * bucket runs its Poisson draw and alias build as a concurrent branch, and
 * the same one persistent z sweep follows.  In the per-bucket mode each
 * bucket runs Poisson draw -> alias build -> z sweep as a concurrent branch
 * with its own launch shapes.  All modes give the same chains bit for bit.
 *
 * Handles are independent of each other and of the single-model state of
 * gpulda.h.  Calls on one handle come from one host thread.  Errors follow
 * gpulda.h (return codes; the fatal-error mode applies).
 */
#ifndef GPULDA_BATCH_H
#define GPULDA_BATCH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One problem: a model and its corpus.  The host arrays are read during
 * gpulda_batch_create only. */
typedef struct GpuldaProblem {
  float alpha;
  float beta;
  uint32_t K;              /* 1 .. GPULDA_BATCH_MAX_K */
  uint32_t V;
  const uint32_t* C;       /* V word counts (initial counts, as Args.C) */
  const uint32_t* z;       /* n_tokens initial topics */
  const uint32_t* w;       /* n_tokens word ids < V */
  const uint32_t* d_len;   /* n_docs document lengths */
  uint64_t n_tokens;
  uint32_t n_docs;
  uint32_t flags;          /* GPULDA_FLAG_LOGLIK */
  uint64_t seed;           /* Philox key, as GpuldaExArgs */
  uint32_t chain;
  uint32_t reserved;
} GpuldaProblem;

#define GPULDA_BATCH_MAX_K 2048u
#define GPULDA_BATCH_BUCKETS 4u

/* Modes (gpulda_batch_set_mode). */
#define GPULDA_BATCH_PER_BUCKET 0u
#define GPULDA_BATCH_MERGED 1u
#define GPULDA_BATCH_MERGED_SWEEP 2u

/* Launch shapes of one K bucket, or of the merged launches. */
typedef struct GpuldaBatchShape {
  uint32_t z_warps_per_block;    /* 2, 4 or 8 documents per block */
  uint32_t z_blocks_per_sm;      /* cap on resident blocks per SM, 0: as many as fit */
  uint32_t phi_cells_per_block;  /* (word, topic) cells per Poisson-draw block */
  uint32_t reserved;
} GpuldaBatchShape;

/* Uploads the problems and draws their initial counts (iteration -1, as
 * initialize does).  *handle receives the batch. */
int gpulda_batch_create(const GpuldaProblem* problems, uint32_t n_problems, void** handle);
int gpulda_batch_destroy(void* handle);

/* Runs n_iter iterations of every problem (graph replays) and waits. */
int gpulda_batch_sweep(void* handle, uint32_t n_iter);

/* Launches the iterations on `cuda_stream` (a cudaStream_t; NULL: the batch's
 * own stream) and returns without waiting, so a caller can time them with its
 * own events.  gpulda_batch_sync waits and checks device status. */
int gpulda_batch_sweep_async(void* handle, uint32_t n_iter, void* cuda_stream);
int gpulda_batch_sync(void* handle);

/* Copies problem p's topics (n_tokens) or counts (V*K, word-major) out. */
int gpulda_batch_read_z(void* handle, uint32_t p, uint32_t* z_out);
int gpulda_batch_read_counts(void* handle, uint32_t p, uint32_t* n_out);

/* Per-problem joint log-likelihood of the last iteration (the formula of
 * gpulda_loglik) into ll[n_problems]; skipped (optional) receives each
 * problem's count of tokens with zero Phi.  Problems without
 * GPULDA_FLAG_LOGLIK report 0. */
int gpulda_batch_loglik(void* handle, double* ll, uint64_t* skipped);

/* Shapes per bucket (GPULDA_BATCH_BUCKETS entries; buckets without problems
 * report zeros).  set_shapes takes effect at the next sweep. */
int gpulda_batch_get_shapes(void* handle, GpuldaBatchShape* shapes);
int gpulda_batch_set_shapes(void* handle, const GpuldaBatchShape* shapes);

/* Selects the mode (GPULDA_BATCH_*) and, if merged_shape is not NULL, the
 * shape of the merged launches (the merged modes' z sweep, and the merged
 * mode's Poisson draw); takes effect at the next sweep. */
int gpulda_batch_set_mode(void* handle, uint32_t mode, const GpuldaBatchShape* merged_shape);

/* Autotuner.  For each bucket without an entry for this device in the cache
 * file, times the candidate shapes on the batch's own data (one Poisson draw
 * and one z sweep per candidate, with the counts and topics restored
 * afterwards, so the chains are unaffected), keeps the fastest and adds it to
 * the cache; buckets with an entry take it from the cache.  Then, unless the
 * cache holds an entry for this batch's composition, it tunes the merged
 * launches' shape the same way, times one whole iteration in each of the
 * three modes and keeps the fastest.  The cache is a JSON object
 * "<device>|sm<count>|K<=<bound>" -> [z_warps_per_block, z_blocks_per_sm,
 * phi_cells_per_block] plus "<device>|sm<count>|merged|<bounds>N~<Mi tokens>"
 * -> [the merged shape, mode]; NULL cache_path tunes without one.
 * n_tuned (optional) receives how many entries were timed. */
int gpulda_batch_tune(void* handle, const char* cache_path, uint32_t* n_tuned);

/* Sizes: [0] problems, [1] tokens, [2] documents, [3] words, [4] cells,
 * [5] device bytes held, [6] buckets in use, [7] iterations run, [8] mode.
 * Returns the number of entries written (<= n). */
int gpulda_batch_info(void* handle, uint64_t* out, int n);

#ifdef __cplusplus
}
#endif

#endif /* GPULDA_BATCH_H */
