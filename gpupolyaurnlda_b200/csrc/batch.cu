// batch.cu -- batched chains (include/gpulda_batch.h): many independent LDA
// problems in shared device arenas, one CUDA graph per iteration.
//
// No counterpart in the reference (one model per process, src/cu/train.cu:
// 16-29).  Every problem runs the same kernels as a solo model -- the batched
// variants differ only in where a problem's parameters and rows are found --
// with problem-local Philox indices, so each chain equals its solo run.
//
// Arenas are laid out bucket by bucket (buckets of K: <= 64, 256, 1024, 2048)
// so that a bucket's cells, words, documents and tokens are contiguous.  The
// iteration graph is
//   bump t; zero S, log-likelihood sums, counters and work counters;
//   merged mode: one launch per stage over every problem --
//     phi_draw_batch over all problems' rows, alias_build_batch over all
//     words, and one z_sweep_kernel<BATCH> whose persistent warps take
//     (problem, document) items longest first from one work queue spanning
//     all buckets, shared memory sized for the largest K;
//   merged-sweep mode (the default): each bucket's phi_draw_batch ->
//     alias_build_batch as concurrent branches, then the one persistent z
//     sweep of the merged mode;
//   per-bucket mode: per bucket, as concurrent branches,
//     phi_draw_batch -> alias_build_batch -> z_sweep_kernel<BATCH>;
// and every kernel reads t from device memory, so the graph is captured once
// and replayed for every iteration.  The autotuner picks launch shapes per
// bucket and for the merged launches, and the fastest mode.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpulda.h"
#include "../../include/gpulda_batch.h"
#include "kernels.cuh"
#include "tables.h"

using namespace gpulda;

namespace {

static_assert(sizeof(GpuldaProblem) == 80, "GpuldaProblem layout");
static_assert(sizeof(GpuldaBatchShape) == 16, "GpuldaBatchShape layout");

constexpr u32 kBucketBound[GPULDA_BATCH_BUCKETS] = {64, 256, 1024, 2048};
constexpr u32 kCellAlign = 32;  // problem row blocks start 128-byte aligned

#define BCK(expr)                                                     \
  do {                                                                \
    cudaError_t e_ = (expr);                                          \
    if (e_ != cudaSuccess) return report_cuda_error(e_, #expr);       \
  } while (0)

__global__ void fill_u32_kernel(u32* p, u64 n, u32 v) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void add_u32_kernel(u32* p, u64 n, u32 add) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] += add;
}

// Per global word w0 + i (i < V): its problem slot and row start.
__global__ void word_rows_kernel(u32* wpid, u64* row_off, u32 w0, u32 V, u32 slot, u64 cell0, u32 K) {
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    wpid[w0 + i] = slot;
    row_off[w0 + i] = cell0 + (u64)i * K;
  }
}

u32 grid_for(u64 n) { return (u32)std::max<u64>(1, std::min<u64>((n + 255) / 256, 4096)); }

u32 bucket_of(u32 K) {
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j)
    if (K <= kBucketBound[j]) return j;
  return GPULDA_BATCH_BUCKETS;
}

struct Bucket {
  bool used = false;
  u32 Kmax = 0;
  u32 slot0 = 0, slot1 = 0;   // problem slots
  u64 cell0 = 0, cell1 = 0;   // arena cells
  u32 word0 = 0, word1 = 0;   // global words
  u64 S0 = 0, S1 = 0;         // per-topic sums
  u32 doc0 = 0, doc1 = 0;     // global documents
  u64 tok0 = 0, tok1 = 0;     // global tokens
  u32 block0 = 0, n_blocks = 0;  // Poisson-draw block table section
  bool want_ll = false;
  GpuldaBatchShape shape{8, 0, 65536, 0};
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

struct Slot {  // one problem, in arena order
  u32 user;    // index in the caller's array
  u32 K, V, n_docs;
  float alpha, beta;
  u32 key0, key1, flags;
  u64 n_tokens;
  u64 cell0, S0, tok0;
  u32 word0, doc0;
};

// Index of the merged launches' work counter (after the buckets').
constexpr u32 kMergedWork = GPULDA_BATCH_BUCKETS;

struct Batch {
  u32 P = 0;
  std::vector<Slot> slots;
  std::vector<u32> slot_of;  // user index -> slot
  Bucket bk[GPULDA_BATCH_BUCKETS];
  // GPULDA_BATCH_*: per-bucket branches, one launch per stage over every
  // problem, or per-bucket Phi/alias branches and one z sweep over every
  // problem's documents
  u32 mode = GPULDA_BATCH_MERGED_SWEEP;
  GpuldaBatchShape mshape{8, 0, 65536, 0};
  u32 Kmax_all = 0;
  bool want_ll_all = false;
  u32 mblock0 = 0, m_n_blocks = 0;  // Poisson-draw block table section of the merged launch
  u32* order_all = nullptr;          // every document, longest first
  u64 cells = 0, N = 0, S_total = 0;
  u32 D = 0, Vtot = 0;
  u64 bytes = 0;
  u64 iters = 0;
  int t = -1;

  std::vector<void*> allocs;
  ModelDev ar{};
  u32 *z = nullptr, *w = nullptr, *d_len = nullptr, *d_idx = nullptr, *order = nullptr;
  u32 *pid = nullptr, *wpid = nullptr;
  u64 *row_off = nullptr;
  u32 *K = nullptr, *key0 = nullptr, *key1 = nullptr;
  float *alpha = nullptr, *beta = nullptr;
  u64 *tok_base = nullptr, *cell_base = nullptr, *S_off = nullptr;
  double *lg_a = nullptr, *lg_Ka = nullptr;
  u32* cdf = nullptr;
  uint8_t* guide = nullptr;
  double* lfac = nullptr;
  uint4* blocks = nullptr;
  u32 blocks_cap = 0;
  u32* t_dev = nullptr;
  double* ll = nullptr;
  unsigned long long* counters = nullptr;
  u32* work = nullptr;
  u32* status = nullptr;

  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;

  template <class T>
  int alloc(T** p, size_t count) {
    *p = nullptr;
    if (!count) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return report_cuda_error(e, "cudaMalloc (batch arenas)");
    allocs.push_back(*p);
    bytes += count * sizeof(T);
    return GPULDA_OK;
  }

  BatchDev zdev() const {
    return BatchDev{pid, row_off, K, alpha, key0, key1, tok_base, lg_a, lg_Ka};
  }
  BatchPhiDev phidev(u32 block0) const {
    return BatchPhiDev{blocks + block0, K, cell_base, S_off, beta, key0, key1, wpid, row_off, cdf, guide, lfac};
  }

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }

  ~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    drop_graph();
    for (auto& b : bk) {
      if (b.s) cudaStreamDestroy(b.s);
      if (b.fork) cudaEventDestroy(b.fork);
      if (b.join) cudaEventDestroy(b.join);
    }
    if (fork) cudaEventDestroy(fork);
    if (stream) cudaStreamDestroy(stream);
    for (void* p : allocs) cudaFree(p);
  }
};

// Poisson-draw block table of bucket j: rows of each problem cut into blocks
// of about `cells` cells.
std::vector<uint4> block_table(const Batch& b, const Bucket& bu, u32 cells) {
  std::vector<uint4> out;
  for (u32 s = bu.slot0; s < bu.slot1; ++s) {
    const Slot& sl = b.slots[s];
    const u32 rows = std::max<u32>(1u, cells / sl.K);
    for (u32 w0 = 0; w0 < sl.V; w0 += rows) out.push_back(make_uint4(s, w0, std::min(sl.V, w0 + rows), 0));
  }
  return out;
}

// Rebuilds every bucket's block table for its current shape, then the merged
// launch's table (every problem) for the merged shape.
int upload_block_tables(Batch& b) {
  std::vector<uint4> all;
  Bucket every;
  every.slot0 = 0;
  every.slot1 = b.P;
  for (auto& bu : b.bk) {
    if (!bu.used) continue;
    std::vector<uint4> t = block_table(b, bu, bu.shape.phi_cells_per_block);
    bu.block0 = (u32)all.size();
    bu.n_blocks = (u32)t.size();
    all.insert(all.end(), t.begin(), t.end());
  }
  {
    std::vector<uint4> t = block_table(b, every, b.mshape.phi_cells_per_block);
    b.mblock0 = (u32)all.size();
    b.m_n_blocks = (u32)t.size();
    all.insert(all.end(), t.begin(), t.end());
  }
  if (all.size() > b.blocks_cap) {
    int rc;
    if ((rc = b.alloc(&b.blocks, all.size()))) return rc;
    b.blocks_cap = (u32)all.size();
  }
  if (!all.empty()) {
    BCK(cudaMemcpyAsync(b.blocks, all.data(), all.size() * sizeof(uint4), cudaMemcpyHostToDevice, b.stream));
    BCK(cudaStreamSynchronize(b.stream));
  }
  return GPULDA_OK;
}

ZLaunch z_args(const Batch& b, u32 j, unsigned long long* counters, double* ll) {
  const Bucket& bu = b.bk[j];
  ZLaunch zl;
  zl.w = b.w;
  zl.z = b.z;
  zl.d_len = b.d_len;
  zl.d_idx = b.d_idx;
  zl.order = b.order + bu.doc0;
  zl.K_d = nullptr;
  zl.n_docs = bu.doc1 - bu.doc0;
  zl.n_tokens = b.N;
  zl.tok_base = 0;
  zl.t = 0;
  zl.t_dev = b.t_dev;
  zl.flags = bu.want_ll ? 1u : 0u;
  zl.counters = counters;
  zl.ll = ll;
  zl.work = b.work + j;
  zl.status = b.status;
  return zl;
}

// The merged launches' z-sweep arguments: every document, longest first.
ZLaunch z_args_merged(const Batch& b, unsigned long long* counters, double* ll) {
  ZLaunch zl = z_args(b, 0, counters, ll);
  zl.order = b.order_all;
  zl.n_docs = b.D;
  zl.flags = b.want_ll_all ? 1u : 0u;
  zl.work = b.work + kMergedWork;
  return zl;
}

// One launch per stage over every problem on stream s (work counter zeroed by
// the caller).
void merged_iteration(const Batch& b, cudaStream_t s) {
  launch_phi_draw_batch(b.ar, b.phidev(b.mblock0), b.m_n_blocks, b.Kmax_all, b.t_dev, s);
  launch_alias_build_batch(b.ar, b.phidev(b.mblock0), b.Kmax_all, 0, b.Vtot, s);
  launch_z_sweep_batch(b.ar, b.zdev(), b.Kmax_all, z_args_merged(b, b.counters, b.ll), s, b.mshape.z_warps_per_block,
                       b.mshape.z_blocks_per_sm);
}

// Each bucket's Phi draw and alias build as concurrent branches (their own
// block sizes and threads per word), then one z sweep over every problem's
// documents on s.
void merged_sweep_iteration(const Batch& b, cudaStream_t s) {
  cudaEventRecord(b.fork, s);
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j) {
    const Bucket& bu = b.bk[j];
    if (!bu.used) continue;
    cudaStreamWaitEvent(bu.s, b.fork, 0);
    launch_phi_draw_batch(b.ar, b.phidev(bu.block0), bu.n_blocks, bu.Kmax, b.t_dev, bu.s);
    launch_alias_build_batch(b.ar, b.phidev(bu.block0), bu.Kmax, bu.word0, bu.word1, bu.s);
    cudaEventRecord(bu.join, bu.s);
    cudaStreamWaitEvent(s, bu.join, 0);
  }
  launch_z_sweep_batch(b.ar, b.zdev(), b.Kmax_all, z_args_merged(b, b.counters, b.ll), s, b.mshape.z_warps_per_block,
                       b.mshape.z_blocks_per_sm);
}

// The bucket's three kernels on stream s (work counter zeroed by the caller).
void bucket_iteration(const Batch& b, u32 j, cudaStream_t s) {
  const Bucket& bu = b.bk[j];
  launch_phi_draw_batch(b.ar, b.phidev(bu.block0), bu.n_blocks, bu.Kmax, b.t_dev, s);
  launch_alias_build_batch(b.ar, b.phidev(bu.block0), bu.Kmax, bu.word0, bu.word1, s);
  launch_z_sweep_batch(b.ar, b.zdev(), bu.Kmax, z_args(b, j, b.counters, b.ll), s, bu.shape.z_warps_per_block,
                       bu.shape.z_blocks_per_sm);
}

int capture_graph(Batch& b) {
  b.drop_graph();
  cudaStream_t s = b.stream;
  BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  launch_bump(b.t_dev, s);
  cudaMemsetAsync(b.ar.S, 0, b.S_total * 8, s);
  cudaMemsetAsync(b.ll, 0, (size_t)b.P * 16, s);
  cudaMemsetAsync(b.counters, 0, kCtrN * 8, s);
  cudaMemsetAsync(b.work, 0, (GPULDA_BATCH_BUCKETS + 1) * 4, s);
  if (b.mode == GPULDA_BATCH_MERGED) {
    merged_iteration(b, s);
  } else if (b.mode == GPULDA_BATCH_MERGED_SWEEP) {
    merged_sweep_iteration(b, s);
  } else {
    cudaEventRecord(b.fork, s);
    for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j) {
      Bucket& bu = b.bk[j];
      if (!bu.used) continue;
      cudaStreamWaitEvent(bu.s, b.fork, 0);
      bucket_iteration(b, j, bu.s);
      cudaEventRecord(bu.join, bu.s);
      cudaStreamWaitEvent(s, bu.join, 0);
    }
  }
  const cudaError_t launch_err = cudaGetLastError();
  cudaGraph_t g = nullptr;
  const cudaError_t end_err = cudaStreamEndCapture(s, &g);
  if (launch_err != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return report_cuda_error(launch_err, "batch iteration capture");
  }
  BCK(end_err);
  b.graph = g;
  BCK(cudaGraphInstantiate(&b.exec, b.graph, 0));
  return GPULDA_OK;
}

int check_status(Batch& b) {
  u32 st = 0;
  BCK(cudaMemcpy(&st, b.status, 4, cudaMemcpyDeviceToHost));
  if (st) {
    BCK(cudaMemset(b.status, 0, 4));
    char buf[96];
    snprintf(buf, sizeof buf, "batched sweep: device status 0x%x", st);
    return report_error(GPULDA_ERR_DEVICE, buf);
  }
  return GPULDA_OK;
}

int validate(const GpuldaProblem& p, u32 i) {
  char buf[160];
  auto bad = [&](int code, const char* what) {
    snprintf(buf, sizeof buf, "batch problem %u: %s", i, what);
    return report_error(code, buf);
  };
  if (p.K < 1 || p.V < 1) return bad(GPULDA_ERR_ARGS, "K and V must be positive");
  if (p.K > GPULDA_BATCH_MAX_K) return bad(GPULDA_ERR_UNSUPPORTED, "K above GPULDA_BATCH_MAX_K");
  if (!(p.alpha > 0.0f) || !(p.beta >= 0.0f) || !std::isfinite(p.alpha) || !std::isfinite(p.beta))
    return bad(GPULDA_ERR_ARGS, "alpha must be > 0 and beta >= 0");
  if (!p.C) return bad(GPULDA_ERR_ARGS, "null word counts");
  if ((p.n_tokens && (!p.z || !p.w)) || (p.n_docs && !p.d_len)) return bad(GPULDA_ERR_ARGS, "null corpus array");
  u64 sum = 0;
  for (u32 d = 0; d < p.n_docs; ++d) {
    if (p.d_len[d] > GPULDA_MAX_DOC_LEN) return bad(GPULDA_ERR_UNSUPPORTED, "document longer than GPULDA_MAX_DOC_LEN");
    sum += p.d_len[d];
  }
  if (sum != p.n_tokens) return bad(GPULDA_ERR_ARGS, "document lengths do not sum to n_tokens");
  for (u64 i2 = 0; i2 < p.n_tokens; ++i2)
    if (p.w[i2] >= p.V || p.z[i2] >= p.K) return bad(GPULDA_ERR_ARGS, "word id >= V or topic >= K");
  return GPULDA_OK;
}

int create_impl(const GpuldaProblem* probs, u32 P, Batch** out) {
  if (!out) return report_error(GPULDA_ERR_ARGS, "null handle pointer");
  *out = nullptr;
  if (!probs || !P) return report_error(GPULDA_ERR_ARGS, "no problems");
  int rc;
  for (u32 i = 0; i < P; ++i)
    if ((rc = validate(probs[i], i))) return rc;

  std::unique_ptr<Batch> holder(new Batch());  // freed on every error return
  Batch& b = *holder;
  b.P = P;
  // arena order: by bucket, then by caller order
  std::vector<u32> perm(P);
  for (u32 i = 0; i < P; ++i) perm[i] = i;
  std::stable_sort(perm.begin(), perm.end(),
                   [&](u32 x, u32 y) { return bucket_of(probs[x].K) < bucket_of(probs[y].K); });
  b.slot_of.resize(P);
  u64 cells = 0, S = 0, N = 0, D = 0, W = 0;
  for (u32 s = 0; s < P; ++s) {
    const GpuldaProblem& p = probs[perm[s]];
    Slot sl;
    sl.user = perm[s];
    sl.K = p.K;
    sl.V = p.V;
    sl.n_docs = p.n_docs;
    sl.alpha = p.alpha;
    sl.beta = p.beta;
    sl.key0 = (u32)p.seed;
    sl.key1 = p.chain;
    sl.flags = p.flags;
    sl.n_tokens = p.n_tokens;
    sl.cell0 = cells;
    sl.S0 = S;
    sl.tok0 = N;
    sl.word0 = (u32)W;
    sl.doc0 = (u32)D;
    cells += ((u64)p.K * p.V + kCellAlign - 1) / kCellAlign * kCellAlign;
    S += p.K;
    N += p.n_tokens;
    D += p.n_docs;
    W += p.V;
    if (N >= (1ull << 32) || D >= (1ull << 32) || W >= (1ull << 32))
      return report_error(GPULDA_ERR_UNSUPPORTED, "batch above 2^32 tokens, documents or words");
    b.slot_of[perm[s]] = s;
    b.slots.push_back(sl);
    Bucket& bu = b.bk[bucket_of(p.K)];
    if (!bu.used) {
      bu.used = true;
      bu.slot0 = s;
      bu.cell0 = sl.cell0;
      bu.word0 = sl.word0;
      bu.S0 = sl.S0;
      bu.doc0 = sl.doc0;
      bu.tok0 = sl.tok0;
    }
    bu.slot1 = s + 1;
    bu.cell1 = cells;
    bu.word1 = (u32)W;
    bu.S1 = S;
    bu.doc1 = (u32)D;
    bu.tok1 = N;
    bu.Kmax = std::max(bu.Kmax, p.K);
    bu.want_ll = bu.want_ll || (p.flags & GPULDA_FLAG_LOGLIK);
    b.Kmax_all = std::max(b.Kmax_all, p.K);
    b.want_ll_all = b.want_ll_all || (p.flags & GPULDA_FLAG_LOGLIK);
  }
  b.cells = cells;
  b.S_total = S;
  b.N = N;
  b.D = (u32)D;
  b.Vtot = (u32)W;

  BCK(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  BCK(cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming));
  for (auto& bu : b.bk) {
    if (!bu.used) continue;
    BCK(cudaStreamCreateWithFlags(&bu.s, cudaStreamNonBlocking));
    BCK(cudaEventCreateWithFlags(&bu.fork, cudaEventDisableTiming));
    BCK(cudaEventCreateWithFlags(&bu.join, cudaEventDisableTiming));
  }
  ModelDev& ar = b.ar;
  ar.V = b.Vtot;
  if ((rc = b.alloc(&ar.n, cells)) || (rc = b.alloc(&ar.q, cells)) || (rc = b.alloc(&ar.al, cells)) ||
      (rc = b.alloc(&ar.csr, cells)) || (rc = b.alloc(&ar.A, W)) || (rc = b.alloc(&ar.S, S)) ||
      (rc = b.alloc(&ar.nnz, W)) || (rc = b.alloc(&b.z, N)) || (rc = b.alloc(&b.w, N)) ||
      (rc = b.alloc(&b.d_len, D)) || (rc = b.alloc(&b.d_idx, D)) || (rc = b.alloc(&b.order, D)) ||
      (rc = b.alloc(&b.order_all, D)) ||
      (rc = b.alloc(&b.pid, D)) || (rc = b.alloc(&b.wpid, W)) || (rc = b.alloc(&b.row_off, W)) ||
      (rc = b.alloc(&b.K, P)) || (rc = b.alloc(&b.key0, P)) || (rc = b.alloc(&b.key1, P)) ||
      (rc = b.alloc(&b.alpha, P)) || (rc = b.alloc(&b.beta, P)) || (rc = b.alloc(&b.tok_base, P)) ||
      (rc = b.alloc(&b.cell_base, P)) || (rc = b.alloc(&b.S_off, P)) || (rc = b.alloc(&b.lg_a, P)) ||
      (rc = b.alloc(&b.lg_Ka, P)) || (rc = b.alloc(&b.cdf, (size_t)P * kPoisN * kPoisW)) ||
      (rc = b.alloc(&b.guide, (size_t)P * kPoisN * 256)) || (rc = b.alloc(&b.lfac, (size_t)P * kLogFacN)) ||
      (rc = b.alloc(&b.t_dev, 1)) || (rc = b.alloc(&b.ll, 2 * (size_t)P)) || (rc = b.alloc(&b.counters, kCtrN)) ||
      (rc = b.alloc(&b.work, GPULDA_BATCH_BUCKETS + 1)) || (rc = b.alloc(&b.status, 1)))
    return rc;

  // Every upload is ordered on the batch stream: a pageable cudaMemcpy may
  // return before its data lands, and kernels on a non-blocking stream would
  // not wait for it.
  // per-problem scalars and tables
  std::vector<u32> hK(P), hk0(P), hk1(P);
  std::vector<float> ha(P), hb(P);
  std::vector<u64> htok(P), hcell(P), hS(P);
  std::vector<double> hlga(P), hlgKa(P);
  std::vector<u32> cdf((size_t)kPoisN * kPoisW);
  std::vector<uint8_t> guide((size_t)kPoisN * 256);
  std::vector<double> lfac(kLogFacN);
  build_log_factorials(kLogFacN, lfac.data());
  for (u32 s = 0; s < P; ++s) {
    const Slot& sl = b.slots[s];
    hK[s] = sl.K;
    hk0[s] = sl.key0;
    hk1[s] = sl.key1;
    ha[s] = sl.alpha;
    hb[s] = sl.beta;
    htok[s] = sl.tok0;
    hcell[s] = sl.cell0;
    hS[s] = sl.S0;
    hlga[s] = std::lgamma((double)sl.alpha);
    hlgKa[s] = std::lgamma((double)sl.K * (double)sl.alpha);
    build_poisson_tables(sl.beta, kPoisN, kPoisW, cdf.data(), guide.data());
    BCK(cudaMemcpyAsync(b.cdf + (size_t)s * kPoisN * kPoisW, cdf.data(), cdf.size() * 4, cudaMemcpyHostToDevice, b.stream));
    BCK(cudaMemcpyAsync(b.guide + (size_t)s * kPoisN * 256, guide.data(), guide.size(), cudaMemcpyHostToDevice, b.stream));
    BCK(cudaMemcpyAsync(b.lfac + (size_t)s * kLogFacN, lfac.data(), lfac.size() * 8, cudaMemcpyHostToDevice, b.stream));
  }
  BCK(cudaMemcpyAsync(b.K, hK.data(), P * 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.key0, hk0.data(), P * 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.key1, hk1.data(), P * 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.alpha, ha.data(), P * 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.beta, hb.data(), P * 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.tok_base, htok.data(), P * 8, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.cell_base, hcell.data(), P * 8, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.S_off, hS.data(), P * 8, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.lg_a, hlga.data(), P * 8, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemcpyAsync(b.lg_Ka, hlgKa.data(), P * 8, cudaMemcpyHostToDevice, b.stream));

  // corpus: tokens with global word ids, document lengths, offsets, owners
  cudaStream_t s = b.stream;
  u32* Cdev = nullptr;
  if ((rc = b.alloc(&Cdev, W))) return rc;
  std::vector<u32> didx(D);
  for (u32 si = 0; si < P; ++si) {
    const Slot& sl = b.slots[si];
    const GpuldaProblem& p = probs[sl.user];
    if (sl.n_tokens) {
      BCK(cudaMemcpyAsync(b.z + sl.tok0, p.z, sl.n_tokens * 4, cudaMemcpyHostToDevice, b.stream));
      BCK(cudaMemcpyAsync(b.w + sl.tok0, p.w, sl.n_tokens * 4, cudaMemcpyHostToDevice, b.stream));
      if (sl.word0) add_u32_kernel<<<grid_for(sl.n_tokens), 256, 0, s>>>(b.w + sl.tok0, sl.n_tokens, sl.word0);
    }
    if (sl.n_docs) {
      BCK(cudaMemcpyAsync(b.d_len + sl.doc0, p.d_len, (size_t)sl.n_docs * 4, cudaMemcpyHostToDevice, b.stream));
      fill_u32_kernel<<<grid_for(sl.n_docs), 256, 0, s>>>(b.pid + sl.doc0, sl.n_docs, si);
      u64 off = sl.tok0;
      for (u32 d = 0; d < sl.n_docs; ++d) {
        didx[sl.doc0 + d] = (u32)off;
        off += p.d_len[d];
      }
    }
    word_rows_kernel<<<grid_for(sl.V), 256, 0, s>>>(b.wpid, b.row_off, sl.word0, sl.V, si, sl.cell0, sl.K);
    BCK(cudaMemcpyAsync(Cdev + sl.word0, p.C, (size_t)sl.V * 4, cudaMemcpyHostToDevice, b.stream));
    const PoisTables tb{b.cdf + (size_t)si * kPoisN * kPoisW, b.guide + (size_t)si * kPoisN * 256,
                        b.lfac + (size_t)si * kLogFacN};
    launch_init_counts_raw(b.ar.n + sl.cell0, sl.K, sl.V, Cdev + sl.word0, tb, sl.beta, sl.key0, sl.key1, s);
  }
  BCK(cudaGetLastError());
  if (D) BCK(cudaMemcpyAsync(b.d_idx, didx.data(), (size_t)D * 4, cudaMemcpyHostToDevice, b.stream));
  // per bucket: documents longest first (stable)
  std::vector<u32> order(D);
  for (auto& bu : b.bk) {
    if (!bu.used) continue;
    std::vector<std::pair<u32, u32>> len;  // (length, doc)
    for (u32 si = bu.slot0; si < bu.slot1; ++si) {
      const Slot& sl = b.slots[si];
      const GpuldaProblem& p = probs[sl.user];
      for (u32 d = 0; d < sl.n_docs; ++d) len.emplace_back(p.d_len[d], sl.doc0 + d);
    }
    std::stable_sort(len.begin(), len.end(), [](const std::pair<u32, u32>& x, const std::pair<u32, u32>& y) {
      return x.first > y.first;
    });
    for (size_t i = 0; i < len.size(); ++i) order[bu.doc0 + i] = len[i].second;
  }
  if (D) BCK(cudaMemcpyAsync(b.order, order.data(), (size_t)D * 4, cudaMemcpyHostToDevice, b.stream));
  // every document, longest first (stable), for the merged launch
  std::vector<u32> order_all(D);
  {
    std::vector<u32> lens(D);
    for (u32 si = 0; si < P; ++si) {
      const Slot& sl = b.slots[si];
      const GpuldaProblem& p = probs[sl.user];
      for (u32 d = 0; d < sl.n_docs; ++d) lens[sl.doc0 + d] = p.d_len[d];
    }
    for (u32 d = 0; d < D; ++d) order_all[d] = d;
    std::stable_sort(order_all.begin(), order_all.end(), [&](u32 x, u32 y) { return lens[x] > lens[y]; });
  }
  if (D) BCK(cudaMemcpyAsync(b.order_all, order_all.data(), (size_t)D * 4, cudaMemcpyHostToDevice, b.stream));
  static const u32 t0 = 0xffffffffu;  // the first bump makes it iteration 0
  BCK(cudaMemcpyAsync(b.t_dev, &t0, 4, cudaMemcpyHostToDevice, b.stream));
  BCK(cudaMemsetAsync(b.status, 0, 4, b.stream));
  BCK(cudaMemsetAsync(b.ll, 0, (size_t)P * 16, b.stream));
  BCK(cudaMemsetAsync(b.counters, 0, kCtrN * 8, b.stream));
  BCK(cudaStreamSynchronize(s));
  // C is needed only for the initial counts
  cudaFree(Cdev);
  b.allocs.erase(std::find(b.allocs.begin(), b.allocs.end(), (void*)Cdev));
  b.bytes -= (u64)W * 4;
  if ((rc = upload_block_tables(b))) return rc;
  *out = holder.release();
  return GPULDA_OK;
}

// --- autotuner ----------------------------------------------------------------

std::string device_key() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  char buf[300];
  snprintf(buf, sizeof buf, "%s|sm%d", prop.name, prop.multiProcessorCount);
  for (char* c = buf; *c; ++c)
    if (*c == '"' || *c == '\\') *c = '_';
  return buf;
}

typedef std::map<std::string, std::vector<unsigned long>> TuneCache;

// Reads "key": [a, b, c] entries of a flat JSON object; anything else is skipped.
TuneCache read_cache(const char* path) {
  TuneCache c;
  if (!path) return c;
  FILE* f = fopen(path, "rb");
  if (!f) return c;
  std::string txt;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, n);
  fclose(f);
  size_t i = 0;
  while ((i = txt.find('"', i)) != std::string::npos) {
    const size_t j = txt.find('"', i + 1);
    if (j == std::string::npos) break;
    const std::string key = txt.substr(i + 1, j - i - 1);
    size_t k = j + 1;
    while (k < txt.size() && (txt[k] == ' ' || txt[k] == ':' || txt[k] == '\n' || txt[k] == '\t')) ++k;
    if (k < txt.size() && txt[k] == '[') {
      const size_t e = txt.find(']', k);
      if (e == std::string::npos) break;
      std::vector<unsigned long> v;
      const char* p = txt.c_str() + k + 1;
      const char* end = txt.c_str() + e;
      while (p < end) {
        char* q = nullptr;
        const unsigned long x = strtoul(p, &q, 10);
        if (q == p) {
          ++p;
          continue;
        }
        v.push_back(x);
        p = q;
      }
      c[key] = v;
      i = e + 1;
    } else {
      i = j + 1;
    }
  }
  return c;
}

bool write_cache(const char* path, const TuneCache& c) {
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) return false;
  fprintf(f, "{\n");
  size_t i = 0;
  for (const auto& kv : c) {
    fprintf(f, "  \"%s\": [", kv.first.c_str());
    for (size_t j = 0; j < kv.second.size(); ++j) fprintf(f, "%s%lu", j ? ", " : "", kv.second[j]);
    fprintf(f, "]%s\n", ++i < c.size() ? "," : "");
  }
  fprintf(f, "}\n");
  const bool ok = fclose(f) == 0;
  return ok && rename(tmp.c_str(), path) == 0;
}

// Device time (ms) of fn() on stream s.
template <class F>
int time_on(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, F fn, float* ms) {
  BCK(cudaEventRecord(e0, s));
  fn();
  BCK(cudaGetLastError());
  BCK(cudaEventRecord(e1, s));
  BCK(cudaEventSynchronize(e1));
  BCK(cudaEventElapsedTime(ms, e0, e1));
  return GPULDA_OK;
}

// Times the candidates of bucket j on the batch's own data and keeps the
// fastest.  Counts and topics of the bucket are saved first and restored at
// the end; the other buckets are untouched.  The iteration counter is set to
// the next iteration for the trial draws and restored.
int tune_bucket(Batch& b, u32 j) {
  Bucket& bu = b.bk[j];
  cudaStream_t s = b.stream;
  const u64 cells = bu.cell1 - bu.cell0, toks = bu.tok1 - bu.tok0;
  u32 *n_save = nullptr, *z_save = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = GPULDA_OK;
  BCK(cudaMalloc(&n_save, std::max<u64>(1, cells) * 4));
  if (cudaMalloc(&z_save, std::max<u64>(1, toks) * 4) != cudaSuccess) {
    cudaFree(n_save);
    return report_error(GPULDA_ERR_NOMEM, "autotuner snapshot");
  }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  u32* n_b = b.ar.n + bu.cell0;
  u32* z_b = b.z + bu.tok0;
  const u32 t_next = (u32)(b.t + 1);
  const GpuldaBatchShape keep = bu.shape;
  GpuldaBatchShape best = keep;
  float best_phi = 1e30f, best_z = 1e30f;
  auto run = [&]() -> int {
    BCK(cudaMemcpyAsync(n_save, n_b, cells * 4, cudaMemcpyDeviceToDevice, s));
    BCK(cudaMemcpyAsync(z_save, z_b, toks * 4, cudaMemcpyDeviceToDevice, s));
    BCK(cudaMemcpyAsync(b.t_dev, &t_next, 4, cudaMemcpyHostToDevice, s));
    BCK(cudaStreamSynchronize(s));
    // Poisson draw: cells per block
    const u32 phi_c[] = {16384, 65536, 262144};
    for (u32 c : phi_c) {
      bu.shape.phi_cells_per_block = c;
      if ((rc = upload_block_tables(b))) return rc;
      BCK(cudaMemcpyAsync(n_b, n_save, cells * 4, cudaMemcpyDeviceToDevice, s));
      BCK(cudaMemsetAsync(b.ar.S + bu.S0, 0, (bu.S1 - bu.S0) * 8, s));
      float ms = 0;
      if ((rc = time_on(s, e0, e1, [&] {
             launch_phi_draw_batch(b.ar, b.phidev(bu.block0), bu.n_blocks, bu.Kmax, b.t_dev, s);
           }, &ms)))
        return rc;
      if (ms < best_phi) {
        best_phi = ms;
        best.phi_cells_per_block = c;
      }
    }
    launch_alias_build_batch(b.ar, b.phidev(bu.block0), bu.Kmax, bu.word0, bu.word1, s);
    BCK(cudaGetLastError());
    // z sweep: documents per block and blocks per SM
    const u32 zc[][2] = {{8, 0}, {4, 0}, {2, 0}, {8, 2}, {4, 4}};
    for (const auto& c : zc) {
      BCK(cudaMemcpyAsync(z_b, z_save, toks * 4, cudaMemcpyDeviceToDevice, s));
      BCK(cudaMemsetAsync(n_b, 0, cells * 4, s));
      BCK(cudaMemsetAsync(b.work + j, 0, 4, s));
      ZLaunch zl = z_args(b, j, b.counters, nullptr);
      zl.flags = 0;
      float ms = 0;
      if ((rc = time_on(s, e0, e1, [&] { launch_z_sweep_batch(b.ar, b.zdev(), bu.Kmax, zl, s, c[0], c[1]); }, &ms)))
        return rc;
      if (ms < best_z) {
        best_z = ms;
        best.z_warps_per_block = c[0];
        best.z_blocks_per_sm = c[1];
      }
    }
    return GPULDA_OK;
  };
  rc = run();
  // restore the chain's state whatever happened
  cudaMemcpyAsync(n_b, n_save, cells * 4, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(z_b, z_save, toks * 4, cudaMemcpyDeviceToDevice, s);
  const u32 t_cur = (u32)b.t;
  cudaMemcpyAsync(b.t_dev, &t_cur, 4, cudaMemcpyHostToDevice, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(n_save);
  cudaFree(z_save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  bu.shape = rc ? keep : best;
  const int rc2 = upload_block_tables(b);
  if (rc) return rc;
  if (e != cudaSuccess) return report_cuda_error(e, "autotuner restore");
  return rc2;
}

// Tunes the merged launches' shape on the batch's own data, then times one
// whole iteration in each of the three modes and keeps the fastest.  All counts and topics
// are saved first and restored at the end, and the iteration counter is put
// back, so the chains are unaffected.
int tune_merged(Batch& b) {
  cudaStream_t s = b.stream;
  u32 *n_save = nullptr, *z_save = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = GPULDA_OK;
  BCK(cudaMalloc(&n_save, std::max<u64>(1, b.cells) * 4));
  if (cudaMalloc(&z_save, std::max<u64>(1, b.N) * 4) != cudaSuccess) {
    cudaFree(n_save);
    return report_error(GPULDA_ERR_NOMEM, "autotuner snapshot");
  }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const u32 t_next = (u32)(b.t + 1), t_cur = (u32)b.t;
  const GpuldaBatchShape keep = b.mshape;
  const u32 keep_mode = b.mode;
  GpuldaBatchShape best = keep;
  u32 best_mode = keep_mode;
  float best_phi = 1e30f, best_z = 1e30f;
  auto restore = [&]() -> int {
    BCK(cudaMemcpyAsync(b.ar.n, n_save, b.cells * 4, cudaMemcpyDeviceToDevice, s));
    BCK(cudaMemcpyAsync(b.z, z_save, b.N * 4, cudaMemcpyDeviceToDevice, s));
    return GPULDA_OK;
  };
  auto run = [&]() -> int {
    BCK(cudaMemcpyAsync(n_save, b.ar.n, b.cells * 4, cudaMemcpyDeviceToDevice, s));
    BCK(cudaMemcpyAsync(z_save, b.z, b.N * 4, cudaMemcpyDeviceToDevice, s));
    BCK(cudaMemcpyAsync(b.t_dev, &t_next, 4, cudaMemcpyHostToDevice, s));
    BCK(cudaStreamSynchronize(s));
    const u32 phi_c[] = {16384, 65536, 262144};
    for (u32 c : phi_c) {
      b.mshape.phi_cells_per_block = c;
      if ((rc = upload_block_tables(b))) return rc;
      if ((rc = restore())) return rc;
      BCK(cudaMemsetAsync(b.ar.S, 0, b.S_total * 8, s));
      float ms = 0;
      if ((rc = time_on(s, e0, e1, [&] {
             launch_phi_draw_batch(b.ar, b.phidev(b.mblock0), b.m_n_blocks, b.Kmax_all, b.t_dev, s);
           }, &ms)))
        return rc;
      if (ms < best_phi) {
        best_phi = ms;
        best.phi_cells_per_block = c;
      }
    }
    launch_alias_build_batch(b.ar, b.phidev(b.mblock0), b.Kmax_all, 0, b.Vtot, s);
    BCK(cudaGetLastError());
    const u32 zc[][2] = {{8, 0}, {4, 0}, {2, 0}, {8, 2}, {4, 4}};
    for (const auto& c : zc) {
      BCK(cudaMemcpyAsync(b.z, z_save, b.N * 4, cudaMemcpyDeviceToDevice, s));
      BCK(cudaMemsetAsync(b.ar.n, 0, b.cells * 4, s));
      BCK(cudaMemsetAsync(b.work + kMergedWork, 0, 4, s));
      ZLaunch zl = z_args_merged(b, b.counters, nullptr);
      zl.flags = 0;
      float ms = 0;
      if ((rc = time_on(s, e0, e1, [&] { launch_z_sweep_batch(b.ar, b.zdev(), b.Kmax_all, zl, s, c[0], c[1]); },
                        &ms)))
        return rc;
      if (ms < best_z) {
        best_z = ms;
        best.z_warps_per_block = c[0];
        best.z_blocks_per_sm = c[1];
      }
    }
    // one whole iteration in each mode, from the same state
    b.mshape = best;
    if ((rc = upload_block_tables(b))) return rc;
    float mode_ms[3] = {1e30f, 1e30f, 1e30f};
    for (u32 m = 0; m < 3; ++m) {
      b.mode = m;
      b.drop_graph();
      if ((rc = capture_graph(b))) return rc;
      if ((rc = restore())) return rc;
      BCK(cudaMemcpyAsync(b.t_dev, &t_cur, 4, cudaMemcpyHostToDevice, s));  // the graph bumps it to t + 1
      if ((rc = time_on(s, e0, e1, [&] { cudaGraphLaunch(b.exec, s); }, &mode_ms[m]))) return rc;
    }
    best_mode = 0;
    for (u32 m = 1; m < 3; ++m)
      if (mode_ms[m] < mode_ms[best_mode]) best_mode = m;
    return GPULDA_OK;
  };
  rc = run();
  restore();
  cudaMemcpyAsync(b.t_dev, &t_cur, 4, cudaMemcpyHostToDevice, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(n_save);
  cudaFree(z_save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b.mshape = rc ? keep : best;
  b.mode = rc ? keep_mode : best_mode;
  b.drop_graph();
  const int rc2 = upload_block_tables(b);
  if (rc) return rc;
  if (e != cudaSuccess) return report_cuda_error(e, "autotuner restore");
  return rc2;
}

Batch* as_batch(void* h) { return static_cast<Batch*>(h); }

}  // namespace

extern "C" int gpulda_batch_create(const GpuldaProblem* problems, uint32_t n_problems, void** handle) {
  Batch* b = nullptr;
  const int rc = create_impl(problems, n_problems, &b);
  if (handle) *handle = rc ? nullptr : b;
  return rc;
}

extern "C" int gpulda_batch_destroy(void* handle) {
  delete as_batch(handle);
  return GPULDA_OK;
}

extern "C" int gpulda_batch_sweep_async(void* handle, uint32_t n_iter, void* cuda_stream) {
  Batch* b = as_batch(handle);
  if (!b) return report_error(GPULDA_ERR_ARGS, "null batch handle");
  int rc;
  if (!b->exec && (rc = capture_graph(*b))) return rc;
  cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : b->stream;
  for (u32 i = 0; i < n_iter; ++i) BCK(cudaGraphLaunch(b->exec, s));
  b->t += (int)n_iter;
  b->iters += n_iter;
  return GPULDA_OK;
}

extern "C" int gpulda_batch_sync(void* handle) {
  Batch* b = as_batch(handle);
  if (!b) return report_error(GPULDA_ERR_ARGS, "null batch handle");
  BCK(cudaDeviceSynchronize());
  return check_status(*b);
}

extern "C" int gpulda_batch_sweep(void* handle, uint32_t n_iter) {
  int rc = gpulda_batch_sweep_async(handle, n_iter, nullptr);
  if (rc) return rc;
  return gpulda_batch_sync(handle);
}

extern "C" int gpulda_batch_read_z(void* handle, uint32_t p, uint32_t* z_out) {
  Batch* b = as_batch(handle);
  if (!b || p >= b->P || !z_out) return report_error(GPULDA_ERR_ARGS, "bad batch read_z arguments");
  const Slot& sl = b->slots[b->slot_of[p]];
  BCK(cudaDeviceSynchronize());
  if (sl.n_tokens) BCK(cudaMemcpy(z_out, b->z + sl.tok0, sl.n_tokens * 4, cudaMemcpyDeviceToHost));
  return GPULDA_OK;
}

extern "C" int gpulda_batch_read_counts(void* handle, uint32_t p, uint32_t* n_out) {
  Batch* b = as_batch(handle);
  if (!b || p >= b->P || !n_out) return report_error(GPULDA_ERR_ARGS, "bad batch read_counts arguments");
  const Slot& sl = b->slots[b->slot_of[p]];
  BCK(cudaDeviceSynchronize());
  BCK(cudaMemcpy(n_out, b->ar.n + sl.cell0, (size_t)sl.K * sl.V * 4, cudaMemcpyDeviceToHost));
  return GPULDA_OK;
}

extern "C" int gpulda_batch_loglik(void* handle, double* ll, uint64_t* skipped) {
  Batch* b = as_batch(handle);
  if (!b || !ll) return report_error(GPULDA_ERR_ARGS, "bad batch loglik arguments");
  if (b->iters == 0) return report_error(GPULDA_ERR_STATE, "no completed sweep");
  BCK(cudaDeviceSynchronize());
  std::vector<double> h(2 * (size_t)b->P);
  BCK(cudaMemcpy(h.data(), b->ll, h.size() * 8, cudaMemcpyDeviceToHost));
  for (u32 p = 0; p < b->P; ++p) {
    const u32 s = b->slot_of[p];
    const bool on = b->slots[s].flags & GPULDA_FLAG_LOGLIK;
    ll[p] = on ? h[2 * s] : 0.0;
    if (skipped) skipped[p] = on ? (uint64_t)h[2 * s + 1] : 0;
  }
  return GPULDA_OK;
}

extern "C" int gpulda_batch_get_shapes(void* handle, GpuldaBatchShape* shapes) {
  Batch* b = as_batch(handle);
  if (!b || !shapes) return report_error(GPULDA_ERR_ARGS, "bad batch get_shapes arguments");
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j) shapes[j] = b->bk[j].used ? b->bk[j].shape : GpuldaBatchShape{};
  return GPULDA_OK;
}

extern "C" int gpulda_batch_set_shapes(void* handle, const GpuldaBatchShape* shapes) {
  Batch* b = as_batch(handle);
  if (!b || !shapes) return report_error(GPULDA_ERR_ARGS, "bad batch set_shapes arguments");
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j) {
    if (!b->bk[j].used) continue;
    const GpuldaBatchShape& sh = shapes[j];
    if ((sh.z_warps_per_block != 2 && sh.z_warps_per_block != 4 && sh.z_warps_per_block != 8) ||
        sh.phi_cells_per_block < 1)
      return report_error(GPULDA_ERR_ARGS, "shape: z_warps_per_block must be 2, 4 or 8, phi cells positive");
  }
  BCK(cudaDeviceSynchronize());
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j)
    if (b->bk[j].used) b->bk[j].shape = shapes[j];
  b->drop_graph();
  return upload_block_tables(*b);
}

extern "C" int gpulda_batch_set_mode(void* handle, uint32_t mode, const GpuldaBatchShape* merged_shape) {
  Batch* b = as_batch(handle);
  if (!b || mode > GPULDA_BATCH_MERGED_SWEEP) return report_error(GPULDA_ERR_ARGS, "bad batch set_mode arguments");
  if (merged_shape) {
    const GpuldaBatchShape& sh = *merged_shape;
    if ((sh.z_warps_per_block != 2 && sh.z_warps_per_block != 4 && sh.z_warps_per_block != 8) ||
        sh.phi_cells_per_block < 1)
      return report_error(GPULDA_ERR_ARGS, "shape: z_warps_per_block must be 2, 4 or 8, phi cells positive");
  }
  BCK(cudaDeviceSynchronize());
  b->mode = mode;
  if (merged_shape) b->mshape = *merged_shape;
  b->drop_graph();
  return upload_block_tables(*b);
}

extern "C" int gpulda_batch_tune(void* handle, const char* cache_path, uint32_t* n_tuned) {
  Batch* b = as_batch(handle);
  if (!b) return report_error(GPULDA_ERR_ARGS, "null batch handle");
  BCK(cudaDeviceSynchronize());
  TuneCache cache = read_cache(cache_path);
  const std::string dev = device_key();
  u32 tuned = 0;
  bool changed = false;
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j) {
    Bucket& bu = b->bk[j];
    if (!bu.used) continue;
    const std::string key = dev + "|K<=" + std::to_string(kBucketBound[j]);
    auto it = cache.find(key);
    if (it != cache.end() && it->second.size() >= 3 &&
        (it->second[0] == 2 || it->second[0] == 4 || it->second[0] == 8) && it->second[2] > 0) {
      bu.shape = GpuldaBatchShape{(u32)it->second[0], (u32)it->second[1], (u32)it->second[2], 0};
      continue;
    }
    const int rc = tune_bucket(*b, j);
    if (rc) return rc;
    cache[key] = {bu.shape.z_warps_per_block, bu.shape.z_blocks_per_sm, bu.shape.phi_cells_per_block};
    ++tuned;
    changed = true;
  }
  // the merged launches' shape and the mode, for this batch's composition
  // (bucket bounds present and total size in millions of tokens)
  std::string comp;
  for (u32 j = 0; j < GPULDA_BATCH_BUCKETS; ++j)
    if (b->bk[j].used) comp += std::to_string(kBucketBound[j]) + ",";
  const std::string mkey = dev + "|merged|" + comp + "N~" + std::to_string(b->N >> 20);
  auto it = cache.find(mkey);
  if (it != cache.end() && it->second.size() >= 4 &&
      (it->second[0] == 2 || it->second[0] == 4 || it->second[0] == 8) && it->second[2] > 0) {
    b->mshape = GpuldaBatchShape{(u32)it->second[0], (u32)it->second[1], (u32)it->second[2], 0};
    b->mode = it->second[3] <= GPULDA_BATCH_MERGED_SWEEP ? (u32)it->second[3] : GPULDA_BATCH_MERGED_SWEEP;
  } else {
    const int rc = tune_merged(*b);
    if (rc) return rc;
    cache[mkey] = {b->mshape.z_warps_per_block, b->mshape.z_blocks_per_sm, b->mshape.phi_cells_per_block,
                   (unsigned long)b->mode};
    ++tuned;
    changed = true;
  }
  b->drop_graph();
  int rc = upload_block_tables(*b);
  if (rc) return rc;
  if (changed && cache_path && !write_cache(cache_path, cache))
    return report_error(GPULDA_ERR_ARGS, "cannot write the autotuner cache file");
  if (n_tuned) *n_tuned = tuned;
  return GPULDA_OK;
}

extern "C" int gpulda_batch_info(void* handle, uint64_t* out, int n) {
  Batch* b = as_batch(handle);
  if (!b || !out) return 0;
  u32 used = 0;
  for (auto& bu : b->bk) used += bu.used;
  const uint64_t v[9] = {b->P, b->N, b->D, b->Vtot, b->cells, b->bytes, used, b->iters, b->mode};
  const int m = n < 9 ? n : 9;
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}
