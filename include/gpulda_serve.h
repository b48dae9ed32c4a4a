/*
 * gpulda_serve.h -- fold-in serving: topic mixtures of new documents against
 * a fixed model held on the device (exported by libGPUPolyaUrnLDA.so).
 *
 * No counterpart in the reference; its closest cousin is the z sweep with the
 * count rebuild disabled (sample_topics, src/cu/topics.cu:36-105).  A request
 * is one document (word ids).  Its topics start uniform at random and are
 * resampled for n_iter Gibbs iterations against the fixed Phi (the draw of
 * the training sweep, with the document's own counts and no update of the
 * model); the result is
 *   theta[k] = (m_k + alpha) / (L + K alpha)           (float)
 *   loglik   = sum_i log sum_k theta[k] Phi[k][w_i]    (double; tokens whose
 *              word has no Phi mass are skipped and counted)
 * with Phi[k][w] = q[w][k] / 2^32 the model's fixed-point Phi.  Random numbers
 * are Philox4x32-10 with counter (token index, low 32 bits of the request id,
 * iteration, stream) and key (seed, chain XOR high 32 bits of the id), so a
 * request's result depends only on its id and words: it is the same whether it
 * runs alone or among any other requests.
 *
 * Continuous batching: submit() queues requests; progress() hands out
 * finished requests, then admits queued requests in arrival order while the
 * request pool (device memory reserved at create) has room for their words
 * and topics and a result record is free.  Every request's warp writes its
 * result straight into mapped host memory and flags it, so poll() returns
 * each request as soon as it is done.
 *   GPULDA_SERVE_PERSISTENT: a resident kernel's warps (slots per SM) take
 *     admitted requests from a device queue whenever they finish one, so a
 *     request starts as soon as a warp is free, whatever else is running.
 *     Idle warps leave after 100 ms; the next admission relaunches the kernel.
 *     A handle admits at most 2^32 - 1 requests over its life.
 *   GPULDA_SERVE_LAUNCH: admitted requests are launched in batches of up to
 *     max_batch (one warp per request, longest first) on `slots` streams;
 *     max_batch = 1 is one launch per document.
 *
 * Handles are independent of each other and of the single-model state of
 * gpulda.h.  Calls on one handle come from one host thread.
 */
#ifndef GPULDA_SERVE_H
#define GPULDA_SERVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPULDA_SERVE_PERSISTENT 0u
#define GPULDA_SERVE_LAUNCH 1u

typedef struct GpuldaServeArgs {
  uint32_t n_iter;        /* fold-in iterations per request */
  uint32_t mode;          /* GPULDA_SERVE_PERSISTENT or GPULDA_SERVE_LAUNCH */
  uint32_t slots;         /* persistent: request warps per SM, 1..32 (0: 32);
                             launch: launches in flight (streams), 1..64 */
  uint32_t max_batch;     /* launch mode: requests per launch, 0: no limit */
  uint32_t max_inflight;  /* requests admitted and not yet handed out, 0: 16384 */
  uint32_t chain;         /* Philox key word 1 (XOR high id bits) */
  uint64_t seed;          /* Philox key word 0 (low 32 bits used) */
  uint64_t pool_bytes;    /* device memory for the words and topics of admitted
                             requests, 0: half the free memory at create, at most 32 GiB */
} GpuldaServeArgs;

#define GPULDA_SERVE_MAX_K 2048u

/* Serves the model of gpulda.h's current single-model state: its Phi and
 * alias tables after the last sample_phi (or corpus sweep) are copied, so the
 * model can be released afterwards. */
int gpulda_serve_create(const GpuldaServeArgs* args, void** handle);

/* Serves a model given as fixed-point Phi q (V*K uint32, word-major,
 * q[w][k] = Phi[k][w] * 2^32); builds its dense masses and alias tables on the
 * device exactly as sample_phi does. */
int gpulda_serve_create_from_phi(const GpuldaServeArgs* args, uint32_t K, uint32_t V, float alpha,
                                 const uint32_t* q, void** handle);

int gpulda_serve_destroy(void* handle);

/* Queues n requests: ids[r], lengths[r] and their word ids back to back in
 * words.  The library copies them before returning.  A request longer than
 * GPULDA_MAX_DOC_LEN, with a word id >= V, or larger than the whole pool is
 * rejected (nothing of this call is queued). */
int gpulda_serve_submit(void* handle, uint32_t n, const uint64_t* ids, const uint32_t* lengths,
                        const uint32_t* words);

/* Hands out finished requests and admits queued ones; never waits. */
int gpulda_serve_progress(void* handle);

/* Moves up to max finished results out: ids, theta (K floats each), loglik,
 * skipped tokens, and the completion time (CLOCK_MONOTONIC ns, taken when
 * progress() saw the request's done flag).  Any output pointer except ids may be NULL.
 * *n_out receives the number written. */
int gpulda_serve_poll(void* handle, uint32_t max, uint64_t* ids, float* theta, double* loglik,
                      uint32_t* skipped, uint64_t* done_ns, uint32_t* n_out);

/* progress() until every queued request has finished. */
int gpulda_serve_drain(void* handle);

/* [0] queued, [1] in flight, [2] finished and not yet polled, [3] kernel launches,
 * [4] requests finished in total, [5] pool bytes, [6] pool bytes in use,
 * [7] admissions deferred for lack of pool memory, [8] K, [9] V.
 * Returns the number of entries written (<= n). */
int gpulda_serve_stats(void* handle, uint64_t* out, int n);

#ifdef __cplusplus
}
#endif

#endif /* GPULDA_SERVE_H */
