// gpulda.cu -- the C ABI of libGPUPolyaUrnLDA.so (declared in include/gpulda.h).
//
// Device orchestration for one model per process (reference: the globals and
// entry points of src/cu/train.cu:16-177).  The reference keeps cuBLAS,
// cuRAND states and V separately allocated alias tables; this library keeps
// four contiguous word-major V*K arrays (counts, fixed-point Phi, alias
// entries) plus per-word and per-topic vectors, and no generator state.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpulda.h"
#include "kernels.cuh"
#include "tables.h"

using namespace gpulda;

static_assert(sizeof(Args) == 32, "Args must match src/ffi.rs Args_FFI");
static_assert(offsetof(Args, C) == 16, "Args.C offset");
static_assert(offsetof(Args, buffer_size) == 24, "Args.buffer_size offset");
static_assert(sizeof(Buffer) == 96, "Buffer must match src/buffer.rs");
static_assert(offsetof(Buffer, n_docs) == 32, "Buffer.n_docs offset");
static_assert(offsetof(Buffer, gpu_z) == 40, "Buffer.gpu_z offset");
static_assert(offsetof(Buffer, stream) == 88, "Buffer.stream offset");

namespace {

enum TimerSlot { kTPhi = 0, kTPrep = 1, kTAlias = 2, kTOffsets = 3, kTZ = 4, kTN = 5 };

// A buffer's sweep is split into this many pieces of about equal token counts
// so that copying piece p+1 in and piece p-1 out overlaps sweeping piece p.
constexpr u32 kPieces = 8;
// Piece p ends at kPieceEnd[p] / 32 of the buffer's tokens.  The first piece
// is small because its copy in is the one wait the sweep cannot hide, the last
// because its copy out is the one that follows the whole sweep; the copies
// (about 55 GB/s each way) outrun the sweep in between.
constexpr u32 kPieceEnd[kPieces] = {1, 3, 7, 12, 18, 24, 29, 32};
// A piece's documents of at least this many times its mean length are swept by
// a separate launch on a high-priority stream: the block scheduler then starts
// them as soon as their piece has arrived and a block slot frees, instead of
// behind the earlier pieces' queues, so the longest sequential chains of the
// last pieces do not set the sweep's tail.
constexpr u32 kLongFactor = 4;

constexpr u32 kWorkCounters = 2 + 2 * kPieces;

struct BufCtx {
  cudaStream_t stream = nullptr;  // sweeps
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaStream_t piece[kPieces] = {};  // one stream per piece, so piece sweeps overlap
  cudaStream_t lpiece[kPieces] = {};  // high priority: each piece's long documents
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // [0] order copied, [1] last copy out issued
  cudaEvent_t in[kPieces] = {}, out[kPieces] = {}, lout[kPieces] = {};
  cudaEvent_t offs = nullptr;     // document offsets of the current sweep are ready
  bool used = false;
  u32* order = nullptr;           // device: document processing order
  // Device work counters of this buffer's launches (kWorkCounters), so sweeps
  // of different buffers may be in flight at the same time: [0] whole buffer,
  // [1, 1 + kPieces) pieces, [1 + kPieces] short documents beside a split sweep,
  // [2 + kPieces, 2 + 2 kPieces) the pieces' long documents.
  u32* work = nullptr;
  std::vector<u32> order_host;    // host staging of the order
  // The last host-buffer sweep's document lengths and what was derived from
  // them (pieces, order, long-document counts; on the device: lengths,
  // offsets, order).  Document lengths rarely change between iterations (the
  // reference's are a read-only map), so an equal array reuses all of it.
  bool cache_valid = false;
  std::vector<u32> d_cache;
  u64 cache_tokens = 0;
  u32 dcut[kPieces + 1] = {};
  u64 tcut[kPieces + 1] = {};
  u32 n_long[kPieces] = {};
};

// Documents longest first (counting sort on length, ties in index order), so
// the longest sequential chains start first and the sweep's tail is short.
// The order does not change any result: documents are independent and the
// count rebuild is an integer sum.
void longest_first(const u32* d_len, u32 n, std::vector<u32>& order) {
  order.resize(n);
  u32 max_len = 0;
  for (u32 i = 0; i < n; ++i) max_len = std::max(max_len, d_len[i]);
  std::vector<u32> start((size_t)max_len + 2, 0);
  for (u32 i = 0; i < n; ++i) start[max_len - d_len[i] + 1]++;
  for (size_t b = 1; b < start.size(); ++b) start[b] += start[b - 1];
  for (u32 i = 0; i < n; ++i) order[start[max_len - d_len[i]]++] = i;
}

// Above this many topics a document's counts live in a shared-memory hash map
// (a dense per-document count array would cost 2 K bytes of shared memory per
// warp); documents of at most kShortDoc tokens are swept by one launch with a
// small map per warp, longer ones by a second launch sized for the longest.
constexpr u32 kMapMinK = 2048;
constexpr u32 kShortDoc = 256;

// Documents longer than kShortDoc and at most kMidDoc tokens are swept by a
// launch of their own, sized for them (and with the large-K store's topic
// bitmap); the few longer ones by another.
constexpr u32 kMidDoc = 1024;

// Longest-first order with the short documents (length <= kShortDoc) first:
// their count, the longest length among the rest, and how many of the rest
// are longer than kMidDoc (they come first among them).
struct DocSplit {
  u32 n_short = 0;
  u32 lmax_long = 0;
  u32 n_huge = 0;    // documents longer than kMidDoc (the first of the long ones)
  u32 lmax_mid = 0;  // longest document of at most kMidDoc tokens among the long ones
};

DocSplit split_longest_first(const u32* d_len, u32 n, std::vector<u32>& order, u32 K) {
  longest_first(d_len, n, order);
  DocSplit sp;
  if (K <= kMapMinK) return sp;
  u32 first_short = n;
  for (u32 i = 0; i < n; ++i)
    if (d_len[order[i]] <= kShortDoc) {
      first_short = i;
      break;
    }
  sp.n_short = n - first_short;
  sp.lmax_long = first_short > 0 ? d_len[order[0]] : 0;
  while (sp.n_huge < first_short && d_len[order[sp.n_huge]] > kMidDoc) ++sp.n_huge;
  sp.lmax_mid = sp.n_huge < first_short ? d_len[order[sp.n_huge]] : 0;
  std::rotate(order.begin(), order.begin() + first_short, order.end());
  return sp;
}

struct Model {
  bool live = false;
  int fatal = 1;
  int last_error = GPULDA_OK;

  u32 K = 0, V = 0, buffer_size = 0, max_D = 0;
  float alpha = 0, beta = 0;
  u32 key0 = 0, key1 = 0, flags = 0;
  int t = -1;           // current iteration (sample_phi calls - 1)
  u64 tok_offset = 0;   // global index of the next buffer's first token in the current iteration
  u64 shard_base = 0;   // global index of this process's first token (document sharding)
  bool swept = false;   // a sweep ran since the last sample_phi

  ModelDev dev{};
  u32* C = nullptr;
  u32* cdf = nullptr;
  uint8_t* guide = nullptr;
  double* lfac = nullptr;
  unsigned long long* counters = nullptr;  // kCtrN
  double* ll = nullptr;                     // 2
  u32* work = nullptr;
  u32* status = nullptr;
  void* alias_scratch = nullptr;
  size_t alias_scratch_bytes = 0;

  cudaStream_t stream = nullptr;       // library stream
  cudaStream_t user_stream = nullptr;  // caller-supplied stream, if any
  cudaEvent_t ev[6] = {};
  bool phi_timed = false, z_timed = false;
  cudaEvent_t z_ev[3] = {};
  u32 launches = 0;
  // Recorded on the caller's stream after each allocation-free sweep; the
  // library's own stream work that reads or resets what that sweep writes
  // (counts, statistics, log-likelihood) waits for it.
  cudaEvent_t noalloc_done = nullptr;
  bool noalloc_pending = false;

  // device-resident corpus
  u32 *cz = nullptr, *cw = nullptr, *cd_len = nullptr, *cd_idx = nullptr, *cK_d = nullptr, *corder = nullptr;
  u32 c_docs = 0;
  u64 c_tokens = 0;
  DocSplit c_split;
};

Model g;

const char* kErrNames[] = {"ok",
                           "CUDA runtime error",
                           "invalid model arguments",
                           "call out of protocol order",
                           "buffer exceeds buffer_size / max_D or is malformed",
                           "device allocation failed",
                           "a kernel reported a violated invariant",
                           "size not supported by this build"};

int fail(int code, const char* what) {
  g.last_error = code;
  if (g.fatal) {
    fprintf(stderr, "GPUPolyaUrnLDA error %d (%s): %s\n", code, kErrNames[code], what);
    exit(code);
  }
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
  return fail(e == cudaErrorMemoryAllocation ? GPULDA_ERR_NOMEM : GPULDA_ERR_CUDA, buf);
}

#define CK(expr)                                           \
  do {                                                     \
    cudaError_t e_ = (expr);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr);    \
  } while (0)

cudaStream_t main_stream() { return g.user_stream ? g.user_stream : g.stream; }

template <class T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (!count) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  return GPULDA_OK;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

int check_status() {
  u32 st = 0;
  CK(cudaMemcpy(&st, g.status, sizeof st, cudaMemcpyDeviceToHost));
  if (st) {
    CK(cudaMemset(g.status, 0, sizeof(u32)));
    char buf[200];
    snprintf(buf, sizeof buf, "device status 0x%x (%s%s%s%s)", st, (st & kStatusBadTopic) ? "topic>=K " : "",
             (st & kStatusBadWord) ? "word>=V " : "", (st & kStatusDocRange) ? "document past n_tokens " : "",
             (st & kStatusDocTooLong) ? "document too long " : "");
    return fail(GPULDA_ERR_DEVICE, buf);
  }
  return GPULDA_OK;
}

void free_model() {
  dfree(g.dev.n);
  dfree(g.dev.q);
  dfree(g.dev.al);
  dfree(g.dev.csr);
  dfree(g.dev.A);
  dfree(g.dev.S);
  dfree(g.dev.Sinv);
  dfree(g.dev.nnz);
  dfree(g.C);
  dfree(g.cdf);
  dfree(g.guide);
  dfree(g.lfac);
  dfree(g.counters);
  dfree(g.ll);
  dfree(g.work);
  dfree(g.status);
  dfree(g.alias_scratch);
  dfree(g.cz);
  dfree(g.cw);
  dfree(g.cd_len);
  dfree(g.cd_idx);
  dfree(g.cK_d);
  dfree(g.corder);
  for (auto& e : g.ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : g.z_ev)
    if (e) cudaEventDestroy(e);
  if (g.stream) cudaStreamDestroy(g.stream);
  if (g.noalloc_done) cudaEventDestroy(g.noalloc_done);
  const int fatal = g.fatal;
  g = Model();
  g.fatal = fatal;
}

int validate_args(const Args* a) {
  if (!a) return fail(GPULDA_ERR_ARGS, "null Args");
  if (a->K < 1 || a->V < 1) return fail(GPULDA_ERR_ARGS, "K and V must be positive");
  if (a->K > GPULDA_MAX_K) return fail(GPULDA_ERR_UNSUPPORTED, "K above GPULDA_MAX_K");
  if (!(a->alpha > 0.0f) || !(a->beta >= 0.0f) || !std::isfinite(a->alpha) || !std::isfinite(a->beta))
    return fail(GPULDA_ERR_ARGS, "alpha must be > 0 and beta >= 0");
  if (a->buffer_size < 1 || a->max_D < 1) return fail(GPULDA_ERR_ARGS, "buffer_size and max_D must be positive");
  if (!a->C) return fail(GPULDA_ERR_ARGS, "null word counts C");
  return GPULDA_OK;
}

int init_impl(const Args* args, Buffer* buffers, u32 n_buffers, const GpuldaExArgs* ex) {
  if (g.live) return fail(GPULDA_ERR_STATE, "initialize called twice without cleanup");
  int rc = validate_args(args);
  if (rc) return rc;
  const int fatal = g.fatal;
  g = Model();
  g.fatal = fatal;
  g.K = args->K;
  g.V = args->V;
  g.alpha = args->alpha;
  g.beta = args->beta;
  g.buffer_size = args->buffer_size;
  g.max_D = args->max_D;
  g.key0 = ex ? (u32)ex->seed : 0u;
  g.key1 = ex ? ex->chain : 0u;
  g.flags = ex ? ex->flags : 0u;
  const size_t cells = (size_t)g.K * g.V;

  CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&g.noalloc_done, cudaEventDisableTiming));
  for (auto& e : g.ev) CK(cudaEventCreate(&e));
  for (auto& e : g.z_ev) CK(cudaEventCreate(&e));
  if ((rc = dalloc(&g.dev.n, cells)) || (rc = dalloc(&g.dev.q, cells)) || (rc = dalloc(&g.dev.al, cells)) ||
      (rc = dalloc(&g.dev.csr, cells)) ||
      (rc = dalloc(&g.dev.A, g.V)) || (rc = dalloc(&g.dev.S, g.K)) || (rc = dalloc(&g.dev.Sinv, g.K)) ||
      (rc = dalloc(&g.dev.nnz, g.V)) ||
      (rc = dalloc(&g.C, g.V)) || (rc = dalloc(&g.cdf, (size_t)kPoisN * kPoisW)) ||
      (rc = dalloc(&g.guide, (size_t)kPoisN * 256)) || (rc = dalloc(&g.lfac, kLogFacN)) ||
      (rc = dalloc(&g.counters, kCtrN)) || (rc = dalloc(&g.ll, 2)) || (rc = dalloc(&g.work, 2 + kPieces)) ||
      (rc = dalloc(&g.status, 1))) {
    free_model();
    return rc;
  }
  g.alias_scratch_bytes = alias_build_scratch_bytes(g.K);
  if (g.alias_scratch_bytes && (rc = dalloc((unsigned char**)&g.alias_scratch, g.alias_scratch_bytes))) {
    free_model();
    return rc;
  }
  std::vector<u32> cdf((size_t)kPoisN * kPoisW);
  std::vector<uint8_t> guide((size_t)kPoisN * 256);
  std::vector<double> lfac(kLogFacN);
  build_poisson_tables(g.beta, kPoisN, kPoisW, cdf.data(), guide.data());
  build_log_factorials(kLogFacN, lfac.data());
  CK(cudaMemcpy(g.cdf, cdf.data(), cdf.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.guide, guide.data(), guide.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.lfac, lfac.data(), lfac.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.C, args->C, (size_t)g.V * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(g.status, 0, 4));
  CK(cudaMemset(g.counters, 0, kCtrN * 8));
  CK(cudaMemset(g.ll, 0, 16));
  // A pageable cudaMemcpy may return before its data lands; kernels on the
  // library's non-blocking streams must not start before that.
  CK(cudaDeviceSynchronize());

  g.dev.K = g.K;
  g.dev.V = g.V;
  g.dev.alpha = g.alpha;
  g.dev.beta = g.beta;
  g.dev.key0 = g.key0;
  g.dev.key1 = g.key1;
  g.dev.tables = PoisTables{g.cdf, g.guide, g.lfac};

  for (u32 i = 0; i < n_buffers; ++i) {
    Buffer& b = buffers[i];
    BufCtx* ctx = new BufCtx();
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
    for (auto& ps : ctx->piece) CK(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
    int lo_prio = 0, hi_prio = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
    for (auto& ps : ctx->lpiece) CK(cudaStreamCreateWithPriority(&ps, cudaStreamNonBlocking, hi_prio));
    for (auto& e : ctx->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->offs, cudaEventDisableTiming));
    for (u32 i = 0; i < kPieces; ++i) {
      CK(cudaEventCreateWithFlags(&ctx->in[i], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&ctx->out[i], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&ctx->lout[i], cudaEventDisableTiming));
    }
    cudaStream_t* sp = new cudaStream_t(ctx->stream);
    b.stream = sp;
    b.gpu_rng = ctx;
    u32 *z, *w, *dl, *di, *kd;
    if ((rc = dalloc(&z, g.buffer_size)) || (rc = dalloc(&w, g.buffer_size)) || (rc = dalloc(&dl, g.max_D)) ||
        (rc = dalloc(&di, g.max_D)) || (rc = dalloc(&kd, g.max_D)) || (rc = dalloc(&ctx->order, g.max_D)) || (rc = dalloc(&ctx->work, kWorkCounters)))
      return rc;
    b.gpu_z = z;
    b.gpu_w = w;
    b.gpu_d_len = dl;
    b.gpu_d_idx = di;
    b.gpu_K_d = kd;
  }

  launch_init_counts(g.dev, g.C, g.stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(g.stream));
  g.live = true;
  return GPULDA_OK;
}

// Orders work about to be issued on `s` after the last allocation-free sweep,
// which ran on a stream of the caller's choosing.
int after_noalloc(cudaStream_t s) {
  if (g.noalloc_pending) CK(cudaStreamWaitEvent(s, g.noalloc_done, 0));
  return GPULDA_OK;
}

// Phi step on `s` without a host synchronisation.
int phi_step_async(cudaStream_t s) {
  if (int rc = after_noalloc(s)) return rc;
  g.t += 1;
  g.tok_offset = g.shard_base;
  g.swept = false;
  g.launches = 0;
  CK(cudaEventRecord(g.ev[0], s));
  CK(cudaMemsetAsync(g.dev.S, 0, (size_t)g.K * 8, s));
  CK(cudaMemsetAsync(g.counters, 0, kCtrN * 8, s));
  CK(cudaMemsetAsync(g.ll, 0, 16, s));
  CK(cudaEventRecord(g.ev[1], s));
  launch_phi_draw(g.dev, (u32)g.t, s);
  CK(cudaGetLastError());
  CK(cudaEventRecord(g.ev[2], s));
  launch_alias_build(g.dev, s, g.alias_scratch, g.alias_scratch_bytes);
  CK(cudaGetLastError());
  CK(cudaEventRecord(g.ev[3], s));
  g.launches += 3;  // Poisson draw, topic reciprocals, alias build
  g.phi_timed = true;
  return GPULDA_OK;
}

// One sweep over documents already on the device.
// One z-sweep launch over n_docs documents whose d_len / d_idx / order / K_d
// start at the given pointers; d_idx offsets are relative to z and w, and the
// tokens' Philox indices start at tok_base.
int z_launch(cudaStream_t s, u32* z, const u32* w, const u32* d_len, const u32* d_idx, const u32* order, u32* K_d,
             u32 n_docs, u64 n_tokens, u64 tok_base, u32* work, u32 lmax = 0) {
  CK(cudaMemsetAsync(work, 0, 4, s));
  ZLaunch zl;
  zl.w = w;
  zl.z = z;
  zl.d_len = d_len;
  zl.d_idx = d_idx;
  zl.order = order;
  zl.K_d = K_d;
  zl.n_docs = n_docs;
  zl.n_tokens = n_tokens;
  zl.tok_base = tok_base;
  zl.t = (u32)g.t;
  zl.flags = (g.flags & GPULDA_FLAG_LOGLIK) ? kZFlagLoglik : 0u;
  zl.counters = g.counters;
  zl.ll = g.ll;
  zl.work = work;
  zl.status = g.status;
  bool done = false;
  if (g.K > kMapMinK && lmax)
    done = (g.flags & GPULDA_FLAG_HASHMAP) ? launch_z_sweep_map(g.dev, zl, s, lmax)
                                           : launch_z_sweep_pairs(g.dev, zl, s, lmax);
  if (!done) launch_z_sweep(g.dev, zl, s);
  CK(cudaGetLastError());
  g.launches += 1;
  return GPULDA_OK;
}

// With a split (large K), `order` lists the short documents first.
// `work` holds kWorkCounters zeroed-per-launch counters.
int z_step_async(cudaStream_t s, u32* z, const u32* w, const u32* d_len, u32* d_idx, const u32* order, u32* K_d,
                 u32 n_docs, u64 n_tokens, bool offsets, cudaEvent_t* ev, u32* work, const DocSplit* split = nullptr) {
  CK(cudaEventRecord(ev[0], s));
  if (offsets) {
    launch_doc_offsets(d_len, d_idx, n_docs, s);
    CK(cudaGetLastError());
    g.launches += 1;
  }
  CK(cudaEventRecord(ev[1], s));
  int rc = GPULDA_OK;
  if (split && g.K > kMapMinK) {
    // Documents over kMidDoc tokens, then those over kShortDoc, then the
    // short ones, one launch each on `s`, each sized for its longest.  Run
    // concurrently on two streams the launches competed for whole SMs (each
    // fills the register file at four blocks per SM): at K=10000 over 8e6
    // documents the sweep took 489 ms concurrently with three blocks per SM,
    // 778 ms with four, and 446 ms one after the other with four.
    const u32 n_long = n_docs - split->n_short;
    if (split->n_huge)
      rc = z_launch(s, z, w, d_len, d_idx, order + split->n_short, K_d, split->n_huge, n_tokens, g.tok_offset, work,
                    split->lmax_long);
    if (!rc && n_long > split->n_huge)
      rc = z_launch(s, z, w, d_len, d_idx, order + split->n_short + split->n_huge, K_d, n_long - split->n_huge,
                    n_tokens, g.tok_offset, work + 1, split->lmax_mid);
    if (!rc && split->n_short)
      rc = z_launch(s, z, w, d_len, d_idx, order, K_d, split->n_short, n_tokens, g.tok_offset,
                    work + 1 + kPieces, kShortDoc);
  } else {
    rc = z_launch(s, z, w, d_len, d_idx, order, K_d, n_docs, n_tokens, g.tok_offset, work);
  }
  if (rc) return rc;
  CK(cudaEventRecord(ev[2], s));
  g.tok_offset += n_tokens;
  g.swept = true;
  return GPULDA_OK;
}

// sample_z_async for host buffers: kPieces pieces of whole documents with
// token counts in the proportions of kPieceEnd; piece p's tokens are copied in on the h2d stream,
// swept on the buffer's stream once they have arrived, and copied out on the
// d2h stream once swept.  Token numbering stays buffer-relative, so the result
// does not depend on the split.
int pipelined_sweep(Buffer* b, BufCtx* ctx) {
  const u32 n = b->n_docs;
  const size_t db = (size_t)n * 4;
  cudaStream_t s = ctx->stream;
  u32* const dcut = ctx->dcut;
  u64* const tcut = ctx->tcut;
  u32* const n_long = ctx->n_long;
  u32* gz = (u32*)b->gpu_z;
  u32* gw = (u32*)b->gpu_w;
  u32* gdl = (u32*)b->gpu_d_len;
  u32* gdi = (u32*)b->gpu_d_idx;
  u32* gkd = (u32*)b->gpu_K_d;
  const bool same = ctx->cache_valid && ctx->d_cache.size() == n && ctx->cache_tokens == b->n_tokens &&
                    std::memcmp(ctx->d_cache.data(), b->d, db) == 0;
  if (same) {
    // lengths, offsets and order on the device are those of the last sweep
    CK(cudaEventRecord(g.z_ev[0], s));
    CK(cudaEventRecord(g.z_ev[1], s));
  } else {
    ctx->cache_valid = false;
    dcut[0] = 0;
    tcut[0] = 0;
    u64 cum = 0;
    u32 pc = 1;
    for (u32 i = 0; i < n && pc < kPieces; ++i) {
      cum += b->d[i];
      while (pc < kPieces && cum * 32 >= (u64)b->n_tokens * kPieceEnd[pc - 1]) {
        dcut[pc] = i + 1;
        tcut[pc] = std::min<u64>(cum, b->n_tokens);
        ++pc;
      }
    }
    for (; pc <= kPieces; ++pc) {
      dcut[pc] = n;
      tcut[pc] = b->n_tokens;
    }
    if (ctx->used) CK(cudaEventSynchronize(ctx->ev[0]));
    ctx->order_host.resize(n);
    std::vector<u32> part;
    for (u32 p = 0; p < kPieces; ++p) {
      const u32 nd = dcut[p + 1] - dcut[p];
      longest_first(b->d + dcut[p], nd, part);
      std::copy(part.begin(), part.end(), ctx->order_host.begin() + dcut[p]);
      // the long documents are a prefix of the longest-first order
      const u64 thr = nd ? (u64)kLongFactor * (tcut[p + 1] - tcut[p]) / nd : 0;
      u32 nl = 0;
      while (nl < nd && (u64)b->d[dcut[p] + part[nl]] >= thr && thr > 0) ++nl;
      n_long[p] = nl;
    }
    CK(cudaMemcpyAsync(gdl, b->d, db, cudaMemcpyHostToDevice, s));
    if (b->K_d) CK(cudaMemcpyAsync(gkd, b->K_d, db, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->order, ctx->order_host.data(), db, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(ctx->ev[0], s));
    CK(cudaEventRecord(g.z_ev[0], s));
    launch_doc_offsets(gdl, gdi, n, s);
    CK(cudaGetLastError());
    g.launches += 1;
    CK(cudaEventRecord(g.z_ev[1], s));
    ctx->d_cache.assign(b->d, b->d + n);
    ctx->cache_tokens = b->n_tokens;
    ctx->cache_valid = true;
  }
  CK(cudaEventRecord(ctx->offs, s));
  if (ctx->used) CK(cudaStreamWaitEvent(ctx->h2d, ctx->ev[1], 0));  // the previous copy out has read gpu_z
  const u64 tok_base = g.tok_offset;
  for (u32 p = 0; p < kPieces; ++p) {
    const u64 t0 = tcut[p], t1 = tcut[p + 1];
    if (t1 > t0) {
      CK(cudaMemcpyAsync(gz + t0, b->z + t0, (t1 - t0) * 4, cudaMemcpyHostToDevice, ctx->h2d));
      CK(cudaMemcpyAsync(gw + t0, b->w + t0, (t1 - t0) * 4, cudaMemcpyHostToDevice, ctx->h2d));
    }
    CK(cudaEventRecord(ctx->in[p], ctx->h2d));
    cudaStream_t ps = ctx->piece[p];
    CK(cudaStreamWaitEvent(ps, ctx->in[p], 0));
    CK(cudaStreamWaitEvent(ps, ctx->offs, 0));  // document offsets are ready
    const u32 nd = dcut[p + 1] - dcut[p], nl = n_long[p];
    if (nl) {
      cudaStream_t ls = ctx->lpiece[p];
      CK(cudaStreamWaitEvent(ls, ctx->in[p], 0));
      CK(cudaStreamWaitEvent(ls, ctx->offs, 0));
      const int rc = z_launch(ls, gz, gw, gdl + dcut[p], gdi + dcut[p], ctx->order + dcut[p], gkd + dcut[p], nl,
                              b->n_tokens, tok_base, ctx->work + 2 + kPieces + p);
      if (rc) return rc;
      CK(cudaEventRecord(ctx->lout[p], ls));
    }
    if (nd > nl) {
      const int rc = z_launch(ps, gz, gw, gdl + dcut[p], gdi + dcut[p], ctx->order + dcut[p] + nl, gkd + dcut[p],
                              nd - nl, b->n_tokens, tok_base, ctx->work + 1 + p);
      if (rc) return rc;
    }
    if (nl) CK(cudaStreamWaitEvent(ps, ctx->lout[p], 0));
    CK(cudaEventRecord(ctx->out[p], ps));
    CK(cudaStreamWaitEvent(s, ctx->out[p], 0));
    CK(cudaStreamWaitEvent(ctx->d2h, ctx->out[p], 0));
    if (t1 > t0) CK(cudaMemcpyAsync(b->z + t0, gz + t0, (t1 - t0) * 4, cudaMemcpyDeviceToHost, ctx->d2h));
  }
  CK(cudaEventRecord(g.z_ev[2], s));
  CK(cudaEventRecord(ctx->ev[1], ctx->d2h));
  g.tok_offset += b->n_tokens;
  g.swept = true;
  g.z_timed = true;
  ctx->used = true;
  return GPULDA_OK;
}

}  // namespace

namespace gpulda {
int report_error(int code, const char* what) { return fail(code, what); }
bool current_model(ModelDev* out, int* t) {
  if (!g.live) return false;
  *out = g.dev;
  *t = g.t;
  return true;
}
int report_cuda_error(cudaError_t e, const char* where) { return cuda_fail(e, where); }
}  // namespace gpulda

// ---------------------------------------------------------------------------
// reference ABI
// ---------------------------------------------------------------------------
extern "C" void initialize(Args* args, Buffer* buffers, uint32_t n_buffers) {
  init_impl(args, buffers, n_buffers, nullptr);
}

extern "C" void sample_phi(void) {
  if (!g.live) {
    fail(GPULDA_ERR_STATE, "sample_phi before initialize");
    return;
  }
  cudaStream_t s = main_stream();
  if (phi_step_async(s)) return;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cuda_fail(e, "sample_phi");
    return;
  }
  check_status();
}

extern "C" void sample_z_async(Buffer* b) {
  if (!g.live || g.t < 0) {
    fail(GPULDA_ERR_STATE, "sample_z_async before initialize/sample_phi");
    return;
  }
  if (!b || !b->gpu_rng) {
    fail(GPULDA_ERR_STATE, "buffer was not passed to initialize");
    return;
  }
  if (b->n_tokens > g.buffer_size || b->n_docs > g.max_D) {
    fail(GPULDA_ERR_BUFFER, "buffer exceeds buffer_size or max_D");
    return;
  }
  if (!b->n_docs) return;
  if (!b->z || !b->w || !b->d) {
    fail(GPULDA_ERR_BUFFER, "null host array in buffer");
    return;
  }
  BufCtx* ctx = (BufCtx*)b->gpu_rng;
  if (!g.user_stream && b->n_docs >= 4 * kPieces && g.K <= kMapMinK) {
    pipelined_sweep(b, ctx);
    return;
  }
  cudaStream_t s = g.user_stream ? g.user_stream : ctx->stream;
  const size_t tb = (size_t)b->n_tokens * 4, db = (size_t)b->n_docs * 4;
#define CKV(expr)                          \
  do {                                     \
    cudaError_t e_ = (expr);               \
    if (e_ != cudaSuccess) {               \
      cuda_fail(e_, #expr);                \
      return;                              \
    }                                      \
  } while (0)
  ctx->cache_valid = false;  // the lengths, offsets and order below replace the pipelined sweep's
  CKV(cudaMemcpyAsync(b->gpu_z, b->z, tb, cudaMemcpyHostToDevice, s));
  CKV(cudaMemcpyAsync(b->gpu_w, b->w, tb, cudaMemcpyHostToDevice, s));
  CKV(cudaMemcpyAsync(b->gpu_d_len, b->d, db, cudaMemcpyHostToDevice, s));
  if (b->K_d) CKV(cudaMemcpyAsync(b->gpu_K_d, b->K_d, db, cudaMemcpyHostToDevice, s));
  // This buffer's previous copy out of order_host must finish before it is rewritten.
  if (ctx->used) CKV(cudaEventSynchronize(ctx->ev[0]));
  const DocSplit split = split_longest_first(b->d, b->n_docs, ctx->order_host, g.K);
  CKV(cudaMemcpyAsync(ctx->order, ctx->order_host.data(), db, cudaMemcpyHostToDevice, s));
  CKV(cudaEventRecord(ctx->ev[0], s));
  if (z_step_async(s, (u32*)b->gpu_z, (const u32*)b->gpu_w, (const u32*)b->gpu_d_len, (u32*)b->gpu_d_idx,
                   ctx->order, (u32*)b->gpu_K_d, b->n_docs, b->n_tokens, true, g.z_ev, ctx->work, &split))
    return;
  g.z_timed = true;
  CKV(cudaMemcpyAsync(b->z, b->gpu_z, tb, cudaMemcpyDeviceToHost, s));
  ctx->used = true;
#undef CKV
}

extern "C" void sync_buffer(Buffer* b) {
  if (!g.live || !b || !b->gpu_rng) {
    fail(GPULDA_ERR_STATE, "sync_buffer on an unknown buffer");
    return;
  }
  BufCtx* ctx = (BufCtx*)b->gpu_rng;
  cudaStream_t s = g.user_stream ? g.user_stream : ctx->stream;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->d2h);
  if (e != cudaSuccess) {
    cuda_fail(e, "sync_buffer");
    return;
  }
  check_status();
}

extern "C" void cleanup(Buffer* buffers, uint32_t n_buffers) {
  if (!g.live) {
    fail(GPULDA_ERR_STATE, "cleanup before initialize");
    return;
  }
  cudaDeviceSynchronize();
  for (u32 i = 0; buffers && i < n_buffers; ++i) {
    Buffer& b = buffers[i];
    dfree(b.gpu_z);
    dfree(b.gpu_w);
    dfree(b.gpu_d_len);
    dfree(b.gpu_d_idx);
    dfree(b.gpu_K_d);
    if (b.gpu_rng) {
      BufCtx* ctx = (BufCtx*)b.gpu_rng;
      for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
      if (ctx->offs) cudaEventDestroy(ctx->offs);
      dfree(ctx->work);
      for (u32 k = 0; k < kPieces; ++k) {
        if (ctx->in[k]) cudaEventDestroy(ctx->in[k]);
        if (ctx->out[k]) cudaEventDestroy(ctx->out[k]);
        if (ctx->lout[k]) cudaEventDestroy(ctx->lout[k]);
      }
      if (ctx->stream) cudaStreamDestroy(ctx->stream);
      if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
      if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
      for (auto& ps : ctx->piece)
        if (ps) cudaStreamDestroy(ps);
      for (auto& ps : ctx->lpiece)
        if (ps) cudaStreamDestroy(ps);
      dfree(ctx->order);
      delete ctx;
    }
    delete (cudaStream_t*)b.stream;
    b.gpu_z = b.gpu_w = b.gpu_d_len = b.gpu_d_idx = b.gpu_K_d = b.gpu_rng = b.stream = nullptr;
  }
  free_model();
}

// ---------------------------------------------------------------------------
// additions
// ---------------------------------------------------------------------------
extern "C" int gpulda_last_error(void) {
  const int e = g.last_error;
  g.last_error = GPULDA_OK;
  return e;
}

extern "C" const char* gpulda_error_string(int code) {
  if (code < 0 || code > GPULDA_ERR_UNSUPPORTED) return "unknown error";
  return kErrNames[code];
}

extern "C" void gpulda_set_fatal_errors(int fatal) { g.fatal = fatal ? 1 : 0; }

extern "C" int gpulda_initialize_ex(const Args* args, Buffer* buffers, uint32_t n_buffers, const GpuldaExArgs* ex) {
  const int fatal = g.fatal;
  g.fatal = 0;
  const int rc = init_impl(args, buffers, n_buffers, ex);
  g.fatal = fatal;
  return rc;
}

extern "C" int gpulda_pin_host(void* p, uint64_t bytes, uint32_t flags) {
  if (!p || !bytes) return fail(GPULDA_ERR_ARGS, "gpulda_pin_host: empty range");
  unsigned f = cudaHostRegisterPortable;
  if (flags & GPULDA_PIN_READ_ONLY) f |= cudaHostRegisterReadOnly;
  const cudaError_t e = cudaHostRegister(p, (size_t)bytes, f);
  if (e != cudaSuccess) {
    cudaGetLastError();  // not sticky: the range stays usable unpinned
    return cuda_fail(e, "cudaHostRegister");
  }
  return GPULDA_OK;
}

extern "C" int gpulda_unpin_host(void* p) {
  const cudaError_t e = cudaHostUnregister(p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cuda_fail(e, "cudaHostUnregister");
  }
  return GPULDA_OK;
}

extern "C" int gpulda_set_token_offset(uint64_t first_token) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "set_token_offset before initialize");
  g.shard_base = first_token;
  g.tok_offset = first_token;
  return GPULDA_OK;
}

extern "C" int gpulda_count_table(void** device_ptr, uint64_t* n_cells) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "count_table before initialize");
  if (!device_ptr || !n_cells) return fail(GPULDA_ERR_ARGS, "null output");
  *device_ptr = g.dev.n;
  *n_cells = (uint64_t)g.K * g.V;
  return GPULDA_OK;
}

extern "C" int gpulda_set_stream(void* s) {
  g.user_stream = (cudaStream_t)s;
  return GPULDA_OK;
}

extern "C" int gpulda_loglik(double* out, uint64_t* n_skipped) {
  if (!g.live || !g.swept) return fail(GPULDA_ERR_STATE, "no completed sweep");
  if (!(g.flags & GPULDA_FLAG_LOGLIK)) return fail(GPULDA_ERR_STATE, "model initialized without GPULDA_FLAG_LOGLIK");
  CK(cudaDeviceSynchronize());
  double h[2];
  CK(cudaMemcpy(h, g.ll, 16, cudaMemcpyDeviceToHost));
  if (out) *out = h[0];
  if (n_skipped) *n_skipped = (uint64_t)h[1];
  return GPULDA_OK;
}

extern "C" int gpulda_corpus_load(const uint32_t* z, const uint32_t* w, const uint32_t* d_len, uint32_t n_docs,
                                  uint64_t n_tokens) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "corpus_load before initialize");
  if (!z || !w || !d_len) return fail(GPULDA_ERR_ARGS, "null corpus array");
  if (n_tokens >= (1ull << 32)) return fail(GPULDA_ERR_UNSUPPORTED, "corpus above 2^32 tokens");
  dfree(g.cz);
  dfree(g.cw);
  dfree(g.cd_len);
  dfree(g.cd_idx);
  dfree(g.cK_d);
  dfree(g.corder);
  g.cz = g.cw = g.cd_len = g.cd_idx = g.cK_d = g.corder = nullptr;
  int rc;
  if ((rc = dalloc(&g.cz, n_tokens)) || (rc = dalloc(&g.cw, n_tokens)) || (rc = dalloc(&g.cd_len, n_docs)) ||
      (rc = dalloc(&g.cd_idx, n_docs)) || (rc = dalloc(&g.cK_d, n_docs)) || (rc = dalloc(&g.corder, n_docs)))
    return rc;
  CK(cudaMemcpy(g.cz, z, n_tokens * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.cw, w, n_tokens * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.cd_len, d_len, (size_t)n_docs * 4, cudaMemcpyHostToDevice));
  std::vector<u32> order;
  g.c_split = split_longest_first(d_len, n_docs, order, g.K);
  CK(cudaMemcpy(g.corder, order.data(), (size_t)n_docs * 4, cudaMemcpyHostToDevice));
  CK(cudaDeviceSynchronize());  // uploads complete before non-blocking streams use them
  launch_doc_offsets(g.cd_len, g.cd_idx, n_docs, g.stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(g.stream));
  g.c_docs = n_docs;
  g.c_tokens = n_tokens;
  return GPULDA_OK;
}

extern "C" int gpulda_corpus_sweep(uint32_t n_iter) {
  if (!g.live || !g.cz) return fail(GPULDA_ERR_STATE, "corpus_sweep without a loaded corpus");
  cudaStream_t s = main_stream();
  for (u32 i = 0; i < n_iter; ++i) {
    int rc = phi_step_async(s);
    if (rc) return rc;
    rc = z_step_async(s, g.cz, g.cw, g.cd_len, g.cd_idx, g.corder, g.cK_d, g.c_docs, g.c_tokens, false, g.z_ev, g.work,
                      &g.c_split);
    if (rc) return rc;
    g.z_timed = true;
  }
  CK(cudaStreamSynchronize(s));
  return check_status();
}

extern "C" int gpulda_corpus_count_rebuild(float* ms) {
  if (!g.live || !g.cz) return fail(GPULDA_ERR_STATE, "corpus_count_rebuild without a loaded corpus");
  cudaStream_t s = main_stream();
  if (int rc = after_noalloc(s)) return rc;
  CK(cudaMemsetAsync(g.dev.n, 0, (size_t)g.K * g.V * 4, s));
  CK(cudaEventRecord(g.ev[4], s));
  launch_count_rebuild(g.dev.n, g.cw, g.cz, g.c_tokens, g.K, g.V, g.status, s);
  CK(cudaGetLastError());
  CK(cudaEventRecord(g.ev[5], s));
  CK(cudaStreamSynchronize(s));
  if (ms) CK(cudaEventElapsedTime(ms, g.ev[4], g.ev[5]));
  return check_status();
}

extern "C" int gpulda_corpus_read_z(uint32_t* z_out) {
  if (!g.live || !g.cz) return fail(GPULDA_ERR_STATE, "no corpus loaded");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(z_out, g.cz, g.c_tokens * 4, cudaMemcpyDeviceToHost));
  return GPULDA_OK;
}

extern "C" int gpulda_kernel_times(float* ms, int n) {
  if (!g.live) return 0;
  float v[kTN] = {0, 0, 0, 0, 0};
  if (g.phi_timed) {
    cudaEventSynchronize(g.ev[3]);
    cudaEventElapsedTime(&v[kTPrep], g.ev[0], g.ev[1]);
    cudaEventElapsedTime(&v[kTPhi], g.ev[1], g.ev[2]);
    cudaEventElapsedTime(&v[kTAlias], g.ev[2], g.ev[3]);
  }
  if (g.z_timed) {
    cudaEventSynchronize(g.z_ev[2]);
    cudaEventElapsedTime(&v[kTOffsets], g.z_ev[0], g.z_ev[1]);
    cudaEventElapsedTime(&v[kTZ], g.z_ev[1], g.z_ev[2]);
  }
  int m = n < kTN ? n : kTN;
  for (int i = 0; i < m; ++i) ms[i] = v[i];
  return m;
}

extern "C" int gpulda_counters(uint64_t* out, int n) {
  if (!g.live) return 0;
  unsigned long long h[kCtrN];
  if (cudaDeviceSynchronize() != cudaSuccess) return 0;
  if (cudaMemcpy(h, g.counters, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  uint64_t v[kCtrN + 1];
  for (int i = 0; i < kCtrN; ++i) v[i] = h[i];
  v[kCtrN] = g.launches;
  int m = n < kCtrN + 1 ? n : kCtrN + 1;
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}

extern "C" int gpulda_debug_read(uint32_t* n, uint32_t* q, uint64_t* alias, uint64_t* A, uint64_t* S, uint32_t* nnz) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "debug_read before initialize");
  CK(cudaDeviceSynchronize());
  const size_t cells = (size_t)g.K * g.V;
  if (n) CK(cudaMemcpy(n, g.dev.n, cells * 4, cudaMemcpyDeviceToHost));
  if (q) CK(cudaMemcpy(q, g.dev.q, cells * 4, cudaMemcpyDeviceToHost));
  if (alias) CK(cudaMemcpy(alias, g.dev.al, cells * 8, cudaMemcpyDeviceToHost));
  if (A) CK(cudaMemcpy(A, g.dev.A, (size_t)g.V * 8, cudaMemcpyDeviceToHost));
  if (S) CK(cudaMemcpy(S, g.dev.S, (size_t)g.K * 8, cudaMemcpyDeviceToHost));
  if (nnz) CK(cudaMemcpy(nnz, g.dev.nnz, (size_t)g.V * 4, cudaMemcpyDeviceToHost));
  return GPULDA_OK;
}

extern "C" int gpulda_debug_write_counts(const uint32_t* n) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "debug_write_counts before initialize");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(g.dev.n, n, (size_t)g.K * g.V * 4, cudaMemcpyHostToDevice));
  CK(cudaDeviceSynchronize());
  return GPULDA_OK;
}

extern "C" int gpulda_debug_tables(uint32_t* cdf, double* lfac) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "debug_tables before initialize");
  if (cdf) CK(cudaMemcpy(cdf, g.cdf, (size_t)kPoisN * kPoisW * 4, cudaMemcpyDeviceToHost));
  if (lfac) CK(cudaMemcpy(lfac, g.lfac, (size_t)kLogFacN * 8, cudaMemcpyDeviceToHost));
  return GPULDA_OK;
}

extern "C" int gpulda_debug_philox(const uint32_t* ctr, uint32_t n, uint32_t key0, uint32_t key1, uint32_t* out) {
  if (!n) return GPULDA_OK;
  u32 *dc = nullptr, *dout = nullptr;
  int rc;
  if ((rc = dalloc(&dc, (size_t)n * 4)) || (rc = dalloc(&dout, (size_t)n * 4))) {
    dfree(dc);
    return rc;
  }
  cudaMemcpy(dc, ctr, (size_t)n * 16, cudaMemcpyHostToDevice);
  launch_debug_philox(dc, n, key0, key1, dout, 0);
  cudaError_t e = cudaMemcpy(out, dout, (size_t)n * 16, cudaMemcpyDeviceToHost);
  dfree(dc);
  dfree(dout);
  if (e != cudaSuccess) return cuda_fail(e, "debug_philox");
  return GPULDA_OK;
}

extern "C" int gpulda_debug_poisson(const uint32_t* count, const uint64_t* idx, uint32_t n, uint32_t t,
                                    uint32_t stream, uint32_t key0, uint32_t key1, uint32_t* out) {
  if (!g.live) return fail(GPULDA_ERR_STATE, "debug_poisson before initialize");
  if (!n) return GPULDA_OK;
  u32 *dc = nullptr, *dout = nullptr;
  u64* di = nullptr;
  int rc;
  if ((rc = dalloc(&dc, n)) || (rc = dalloc(&dout, n)) || (rc = dalloc(&di, n))) {
    dfree(dc);
    dfree(dout);
    return rc;
  }
  cudaMemcpy(dc, count, (size_t)n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(di, idx, (size_t)n * 8, cudaMemcpyHostToDevice);
  launch_debug_poisson(g.dev, dc, di, n, t, stream, key0, key1, dout, 0);
  cudaError_t e = cudaMemcpy(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost);
  dfree(dc);
  dfree(dout);
  dfree(di);
  if (e != cudaSuccess) return cuda_fail(e, "debug_poisson");
  return GPULDA_OK;
}

extern "C" int gpulda_debug_alias(const uint32_t* q, uint32_t K, uint64_t* table_out) {
  if (K < 1 || K > 11264) return fail(GPULDA_ERR_UNSUPPORTED, "debug_alias supports 1 <= K <= 11264");
  u32* dq = nullptr;
  u64* dout = nullptr;
  int rc;
  if ((rc = dalloc(&dq, K)) || (rc = dalloc(&dout, K))) {
    dfree(dq);
    return rc;
  }
  cudaMemcpy(dq, q, (size_t)K * 4, cudaMemcpyHostToDevice);
  launch_debug_alias(dq, K, dout, 0);
  cudaError_t e = cudaMemcpy(table_out, dout, (size_t)K * 8, cudaMemcpyDeviceToHost);
  dfree(dq);
  dfree(dout);
  if (e != cudaSuccess) return cuda_fail(e, "debug_alias");
  return GPULDA_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free sweep over documents that are already in device memory.
//
// For callers that may not allocate device memory at the point of the call:
// code that owns all device memory through its own pool, services that must
// not allocate once serving has started, or work issued where cudaMalloc is
// not permitted.  Its only scratch (document offsets and the work-queue
// counter) is the file-scope device array below, sized for
// GPULDA_NOALLOC_MAX_DOCS documents: 4 MiB + 256 B that every GPU which loads
// this library holds until the process exits.  In host code the array's name
// is only a host-side stand-in; its device address is looked up once per
// device with cudaGetSymbolAddress (on the first call on that device, which
// is why that first call should come before any stream capture).  All calls
// share the array, so calls whose work overlaps on the GPU race with each
// other; the work-queue counter is cleared on every call.  Calls issued one
// after another from the host are ordered on the GPU even on different
// streams (each waits for the previous call's event), and the next Phi step
// waits for the last call, so the counts it reads are complete.
// ---------------------------------------------------------------------------
namespace {
constexpr u32 kNoAllocMaxDocs = GPULDA_NOALLOC_MAX_DOCS;
constexpr u32 kNoAllocTail = 64;  // work-queue counter and padding
static __device__ __align__(256) u32 g_noalloc_scratch[kNoAllocMaxDocs + kNoAllocTail];
constexpr int kNoAllocMaxDevices = 64;
u32* g_noalloc_addr[kNoAllocMaxDevices] = {};
}  // namespace

extern "C" int gpulda_sample_z_device_noalloc(uint32_t* z, const uint32_t* w, const uint32_t* d_len,
                                              uint32_t n_docs, uint64_t n_tokens, void* stream) {
  if (!g.live || g.t < 0) return fail(GPULDA_ERR_STATE, "gpulda_sample_z_device_noalloc before initialize/sample_phi");
  if (n_docs > kNoAllocMaxDocs)
    return fail(GPULDA_ERR_UNSUPPORTED,
                "gpulda_sample_z_device_noalloc: n_docs exceeds GPULDA_NOALLOC_MAX_DOCS (1048576 documents)");
  if (n_tokens >= (1ull << 32))
    return fail(GPULDA_ERR_UNSUPPORTED, "gpulda_sample_z_device_noalloc: n_tokens must be below 2^32");
  if (!n_docs) return GPULDA_OK;
  if (!z || !w || !d_len) return fail(GPULDA_ERR_ARGS, "gpulda_sample_z_device_noalloc: null device array");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(GPULDA_ERR_UNSUPPORTED, "gpulda_sample_z_device_noalloc: device ordinal above 63");
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_addr[dev] = (u32*)p;
  }
  u32* d_idx = g_noalloc_addr[dev];
  u32* work = d_idx + kNoAllocMaxDocs;
  cudaStream_t s = stream ? (cudaStream_t)stream : main_stream();
  // the previous call's use of the shared scratch ends before this one's begins
  if (int rc = after_noalloc(s)) return rc;
  CK(cudaMemsetAsync(work, 0, sizeof(u32), s));
  launch_doc_offsets(d_len, d_idx, n_docs, s);
  CK(cudaGetLastError());
  ZLaunch zl;
  zl.w = w;
  zl.z = z;
  zl.d_len = d_len;
  zl.d_idx = d_idx;
  zl.order = nullptr;
  zl.K_d = nullptr;
  zl.n_docs = n_docs;
  zl.n_tokens = n_tokens;
  zl.tok_base = g.tok_offset;
  zl.t = (u32)g.t;
  zl.flags = (g.flags & GPULDA_FLAG_LOGLIK) ? kZFlagLoglik : 0u;
  zl.counters = g.counters;
  zl.ll = g.ll;
  zl.work = work;
  zl.status = g.status;
  // Above kMapMinK topics, the large-K store the other sweeps use.  The
  // lengths are on the device only, so the launch accepts any document length
  // and sizes each document's store for K distinct topics.
  bool done = false;
  if (g.K > kMapMinK)
    done = (g.flags & GPULDA_FLAG_HASHMAP) ? launch_z_sweep_map(g.dev, zl, s, 65535u)
                                           : launch_z_sweep_pairs(g.dev, zl, s, 65535u);
  if (!done) launch_z_sweep(g.dev, zl, s);
  CK(cudaGetLastError());
  CK(cudaEventRecord(g.noalloc_done, s));
  g.noalloc_pending = true;
  g.launches += 2;
  g.tok_offset += n_tokens;
  g.swept = true;
  return GPULDA_OK;
}
