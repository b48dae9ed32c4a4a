// serve.cu -- fold-in serving with continuous batching (include/gpulda_serve.h).
//
// No counterpart in the reference.  A request is one new document; its topic
// mixture is estimated against a fixed model (fixed-point Phi, per-word alias
// tables and nonzero lists, exactly as the training sweep holds them) by
// n_iter Gibbs iterations of the training sweep's per-token draw
// (doc_counts.cuh) without the count rebuild, keyed by the request id.
//
// Every request's warp writes its result record (theta, log-likelihood) into
// a mapped pinned host area and then raises the record's done flag, so the
// host hands each request out the moment it finishes.
//
// Persistent mode (the default): one resident kernel whose warps take
// requests from a device ring as they become free -- the warps are the batch
// slots.  The host publishes admitted requests by copying their words into
// the device request pool, their descriptors into the ring and then the new
// ring tail, all on one copy stream, so a warp that sees the tail finds the
// descriptors and words in place.  Claims are a compare-and-swap on the ring
// head.  Idle warps sleep with exponential backoff and leave after kIdleNs
// without work, or at once when the host raises the stop flag; the host
// relaunches the kernel whenever requests are in flight and none is running.
//
// Launch mode: queued requests are launched in batches (one warp per request,
// longest first) on a ring of streams; max_batch = 1 is one launch per
// document.
#include <time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpulda.h"
#include "../../include/gpulda_serve.h"
#include "doc_counts.cuh"
#include "kernels.cuh"

using namespace gpulda;

namespace {

static_assert(sizeof(GpuldaServeArgs) == 40, "GpuldaServeArgs layout");

#define SCK(expr)                                                 \
  do {                                                            \
    cudaError_t e_ = (expr);                                      \
    if (e_ != cudaSuccess) return report_cuda_error(e_, #expr);   \
  } while (0)

constexpr u32 kMaxSlots = 64;
constexpr u32 kStaging = 8;                     // rotating pinned staging buffers (persistent mode)
constexpr u64 kIdleNs = 100000000ull;           // persistent warps leave after 100 ms without work
constexpr u32 kMaxSleepNs = 32768;              // backoff cap while idle
constexpr u64 kDrainStallNs = 120000000000ull;  // drain gives up after 120 s without progress

u64 align_up(u64 x, u64 a) { return (x + a - 1) / a * a; }

u64 now_ns() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (u64)ts.tv_sec * 1000000000ull + (u64)ts.tv_nsec;
}

// One request on the device (32 bytes): its words and topic scratch (u32
// offsets into the request pool), id, length and result record.
struct FoldReq {
  u64 w_off;
  u64 z_off;
  u64 rid;
  u32 len;
  u32 rec;
};
static_assert(sizeof(FoldReq) == 32, "FoldReq");

// Shared memory per request warp: the document's counts and the staged
// per-token data of a 32-token chunk.
inline size_t fold_smem_bytes(u32 K) { return doc_counts_bytes(K) + 32 * 32; }

// Output record of a request: theta[K] (float), then 8-byte aligned the
// log-likelihood (double), skipped tokens (u32) and the done flag (u32).
__host__ __device__ inline size_t ll_offset(u32 K) { return (size_t)K * 4 + ((K & 1) ? 4 : 0); }
inline u32 record_bytes(u32 K) { return (u32)align_up(ll_offset(K) + 16, 16); }

struct FoldCommon {
  ModelDev m;           // K, V, alpha, q, al, csr, A, nnz
  u32* pool;            // request pool (words, topic scratch, launch descriptors)
  unsigned char* recs;  // result records (mapped host memory)
  u32 rec_bytes;
  u32 n_iter;
  u32 key0, key1;
  u32* status;
  u64 pool_words;  // request pool size (u32 units)
  u32 n_recs;      // result records
};

// Device status bit: a request descriptor pointing outside the pool or the
// records (the request is skipped).
constexpr u32 kStatusBadRequest = 16;

// Fold-in of one request by one warp.  Words are read through L2 only: the
// pool is refilled by copies while kernels run, so an SM's L1 may still hold
// an earlier request's words at the same address.
__device__ void fold_request(const FoldCommon& a, DocCounts& dc, uint4* stage, const FoldReq& rq, u32 lane) {
  if (rq.w_off + rq.len > a.pool_words || rq.z_off + rq.len > a.pool_words || rq.rec >= a.n_recs ||
      rq.len > 65535u) {
    if (lane == 0) atomicOr(a.status, kStatusBadRequest);
    return;
  }
  const ModelDev& m = a.m;
  const u32 K = m.K, V = m.V, L = rq.len;
  const float alpha = m.alpha;
  const u32* w = a.pool + rq.w_off;
  u32* z = a.pool + rq.z_off;
  const u64 ridx = (u64)(u32)rq.rid << 32;  // Philox index: (token, low id bits)
  const u32 k0 = a.key0, k1 = a.key1 ^ (u32)(rq.rid >> 32);
  u32 status = 0;

  for (u32 i = lane; i < L; i += 32) {
    const U4 r = draw4(ridx | i, 0, kStreamFoldInit, 0, k0, k1);
    z[i] = (u32)(((u64)r.x * K) >> 32);
  }
  __syncwarp();
  doc_counts_build(dc, z, L, K, lane, &status, kStatusBadTopic);

  for (u32 t = 0; t < a.n_iter; ++t) {
    for (u32 base = 0; base < L; base += 32) {
      const u32 i = base + lane;
      const bool valid = i < L;
      u32 my_w = valid ? __ldcg(w + i) : 0;
      const u32 my_z = valid ? z[i] : 0;
      if (my_w >= V) {
        status |= kStatusBadWord;
        my_w %= V;
      }
      const U4 r = draw4(ridx | i, t, kStreamFold, 0, k0, k1);
      const u32 my_nw = valid ? __ldg(m.nnz + my_w) : 0u;
      const u64 my_A = valid ? __ldg(m.A + my_w) : 0ull;
      const u32 my_s = (u32)(((u64)r.z * my_nw) >> 32);
      const u64 my_row = (u64)my_w * K;
      const u64 my_al = (valid && my_nw) ? __ldg(m.al + my_row + my_s) : 0ull;
      u32 new_z = my_z;
      const u32 nt = min(32u, L - base);
      // per-token data staged in shared memory (broadcast loads, not shuffles)
      __syncwarp();
      stage[2 * lane] = make_uint4(my_z, r.x, r.y, my_nw);
      stage[2 * lane + 1] = make_uint4((u32)my_row, (u32)(my_row >> 32), (u32)my_A, (u32)(my_A >> 32));
      __syncwarp();
      for (u32 j = 0; j < nt; ++j) {
        const uint4 s0 = stage[2 * j], s1 = stage[2 * j + 1];
        const u32 zj = s0.x, r0 = s0.y, r1 = s0.z, nw = s0.w;
        const size_t row = ((u64)s1.y << 32) | s1.x;
        const u64 Aw = ((u64)s1.w << 32) | s1.z;
        u32 nzm;
        bool sp;
        // as in the training sweep: as few register slots as the walk needs
        const u32 cper_j = ((nw < dc.nl ? nw : dc.nl) + 31) >> 5;
        const u32 k = cper_j <= 2 ? token_step<2u>(dc, zj, r0, r1, r.w, my_al, j, m.q + row, m.csr + row, nw, Aw, alpha,
                                                   lane, &nzm, &sp)
                                  : token_step<4u>(dc, zj, r0, r1, r.w, my_al, j, m.q + row, m.csr + row, nw, Aw, alpha,
                                                   lane, &nzm, &sp);
        if (lane == j) new_z = k;
        __syncwarp();
      }
      if (valid) z[i] = new_z;
      __syncwarp();
    }
  }

  // theta and the log-likelihood of the document's words under it
  unsigned char* rec = a.recs + (size_t)rq.rec * a.rec_bytes;
  float* theta = (float*)rec;
  const double denom = (double)L + (double)K * (double)alpha;
  for (u32 k = lane; k < K; k += 32) theta[k] = (float)(((double)dc.cnt[k] + (double)alpha) / denom);
  // sum_k (m_k + alpha) q[w][k] = sum_k m_k q[w][k] + alpha A[w]: the first term
  // exactly (u64) over the shorter of the two lists, the second from the dense mass
  double ll = 0.0;
  u32 skipped = 0;
  for (u32 i = 0; i < L; ++i) {
    const u32 wi = __ldcg(w + i) % V;
    const u32 nw = __ldg(m.nnz + wi);
    const size_t row = (size_t)wi * K;
    u64 part = 0;
    if (nw < dc.nl) {
      for (u32 e = lane; e < nw; e += 32) {
        const u64 ent = __ldg(m.csr + row + e);
        part += (u64)dc.cnt[(u32)ent & 0xffffu] * (u32)(ent >> 32);
      }
    } else {
      for (u32 e = lane; e < dc.nl; e += 32) {
        const u32 k = dc.tl[e];
        part += (u64)dc.cnt[k] * __ldg(m.q + row + k);
      }
    }
    const u64 Bw = warp_sum_u64(part);
    const double s = (double)Bw + (double)alpha * (double)__ldg(m.A + wi);
    if (s > 0.0)
      ll += log(s);
    else
      ++skipped;
  }
  if (lane == 0) {
    ll -= (double)(L - skipped) * (log(denom) + 22.18070977791825);  // 2^32 fixed point
    *(double*)(rec + ll_offset(K)) = ll;
    *(u32*)(rec + ll_offset(K) + 8) = skipped;
  }
  status = __reduce_or_sync(kFullMask, status);
  if (lane == 0 && status) atomicOr(a.status, status);
  // The record lives in host memory: every lane's writes are made visible to
  // the host before lane 0 raises the flag.
  __threadfence_system();
  __syncwarp();
  if (lane == 0) *(volatile u32*)(rec + ll_offset(K) + 12) = 1u;
  __syncwarp();
}

// Launch mode: one request per block of one warp.
__global__ void __launch_bounds__(32) fold_launch_kernel(FoldCommon a, const FoldReq* items) {
  extern __shared__ __align__(16) unsigned char fsm[];
  DocCounts dc = doc_counts_at(fsm, a.m.K);
  uint4* stage = reinterpret_cast<uint4*>(fsm + doc_counts_bytes(a.m.K));
  const FoldReq rq = items[blockIdx.x];
  fold_request(a, dc, stage, rq, threadIdx.x);
}

struct RingDev {
  const FoldReq* ring;       // cap entries
  u64 cap;                   // power of two
  unsigned long long* head;  // requests claimed
  const u64* tail;           // requests published (written by host copies)
  const u32* stop;           // raised by the host
};

// Polling loads of words that other agents write while the kernel runs: the
// ring tail and the stop flag (host copies) and the ring head (other warps'
// atomics).  Relaxed strong loads read the coherent copy (never a stale L1
// line) without the L1 invalidation an acquire would cost the SM's working
// warps on every poll; a claim is followed by one fence instead.
__device__ __forceinline__ u64 load_relaxed_sys(const u64* p) {
  u64 v;
  asm volatile("ld.relaxed.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ u32 load_relaxed_sys(const u32* p) {
  u32 v;
  asm volatile("ld.relaxed.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ u64 load_relaxed_gpu(const unsigned long long* p) {
  u64 v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Nanoseconds from the GPU's global timer.
__device__ __forceinline__ u64 global_timer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Persistent mode: every block is one warp that serves requests until it has
// been idle for kIdleNs or the stop flag is up.  Every wait is bounded.
__global__ void __launch_bounds__(32, 32) fold_persistent_kernel(FoldCommon a, RingDev q) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const u32 lane = threadIdx.x;
  DocCounts dc = doc_counts_at(fsm, a.m.K);
  uint4* stage = reinterpret_cast<uint4*>(fsm + doc_counts_bytes(a.m.K));
  while (true) {
    unsigned long long mine = ~0ull;
    if (lane == 0) {
      u64 idle_since = 0;
      u32 sleep = 256;
      unsigned long long h = load_relaxed_gpu(q.head);
      while (true) {
        if (load_relaxed_sys(q.stop)) break;
        const u64 t = load_relaxed_sys(q.tail);
        if (h < t) {
          const unsigned long long old = atomicCAS(q.head, h, h + 1);
          if (old == h) {
            mine = h;
            __threadfence_system();  // the entry and words are read after the tail that covers them
            break;
          }
          h = old;  // another warp claimed h
          continue;
        }
        const u64 now = global_timer_ns();
        if (!idle_since) idle_since = now;
        if (now - idle_since > kIdleNs) break;
        __nanosleep(sleep);
        if (sleep < kMaxSleepNs) sleep <<= 1;
        h = load_relaxed_gpu(q.head);
      }
    }
    mine = __shfl_sync(kFullMask, mine, 0);
    if (mine == ~0ull) break;
    // not through L1: ring entries are rewritten by copies
    const uint4* e = reinterpret_cast<const uint4*>(q.ring + (mine & (q.cap - 1)));
    const uint4 lo = __ldcg(e), hi = __ldcg(e + 1);
    FoldReq rq;
    rq.w_off = ((u64)lo.y << 32) | lo.x;
    rq.z_off = ((u64)lo.w << 32) | lo.z;
    rq.rid = ((u64)hi.y << 32) | hi.x;
    rq.len = hi.z;
    rq.rec = hi.w;
    fold_request(a, dc, stage, rq, lane);
  }
}

struct Req {
  u64 id;
  std::vector<u32> words;
};

struct Result {
  u64 id;
  double ll;
  u32 skipped;
  u64 done_ns;
  std::vector<float> theta;
};

struct InFlight {
  u64 id;
  u32 rec;
  u64 extent;  // pool offset of its extent (persistent mode)
};

// Pinned host staging buffer of fixed size, with the event of the copies that
// last read it.  It is allocated once: allocating or freeing pinned memory
// synchronizes the device, which would wait for the resident kernel.
struct Staging {
  unsigned char* p = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  bool pending = false;
  Staging() = default;
  Staging(const Staging&) = delete;
  Staging& operator=(const Staging&) = delete;
  int init(size_t bytes) {
    SCK(cudaHostAlloc((void**)&p, bytes, cudaHostAllocDefault));
    cap = bytes;
    SCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return GPULDA_OK;
  }
  // Waits until the copies that read the buffer last are done.
  int ready() {
    if (pending) {
      SCK(cudaEventSynchronize(ev));
      pending = false;
    }
    return GPULDA_OK;
  }
  ~Staging() {
    if (p) cudaFreeHost(p);
    if (ev) cudaEventDestroy(ev);
  }
};

// Staging bytes needed for n requests with T tokens: a 16-byte header, the
// descriptors, the words.
inline size_t staging_bytes(u64 n, u64 T) { return align_up(16 + n * sizeof(FoldReq), 16) + T * 4; }

// Per staging buffer (persistent mode / launch slot): room for the largest
// request several times over.
constexpr size_t kStagingBytes = 4u << 20, kSlotStagingBytes = 1u << 20;
static_assert(kSlotStagingBytes >= 16 + 32 + 4 * 65535ull, "a staging buffer holds any single request");

struct LaunchSlot {
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  u64 ext_off = 0, ext_words = 0;
  Staging st;
};

struct Server {
  u32 K = 0, V = 0;
  float alpha = 0;
  GpuldaServeArgs args{};
  bool persistent = true;
  u32 rec_bytes = 0, max_inflight = 0;
  size_t stage_cap = 0;  // bytes of each staging buffer
  FoldCommon fc{};
  std::vector<void*> allocs;
  // request pool, u32 units
  u64 pool_words = 0, pool_used = 0;
  std::map<u64, u64> free_ext;           // offset -> size
  std::map<u64, std::pair<u64, u32>> extents;  // persistent mode: offset -> (size, requests not yet out)
  // result records (mapped pinned host memory)
  unsigned char* recs_host = nullptr;
  std::vector<u32> free_recs;
  std::deque<Req> queue;
  std::deque<InFlight> inflight;
  std::deque<Result> results;
  u64 launches = 0, finished = 0, deferred = 0;
  // persistent mode
  cudaStream_t copy_s = nullptr, kern_s = nullptr;
  cudaEvent_t kern_ev = nullptr;
  bool kern_live = false;
  FoldReq* ring = nullptr;
  u64 ring_cap = 0;
  unsigned char* ctl = nullptr;  // device: head (u64) at 0, tail (u64) at 8, stop (u32) at 16
  u64 published = 0;
  std::unique_ptr<Staging[]> staging;
  u32 next_staging = 0;
  u32 resident_per_sm = 32;
  // launch mode
  std::unique_ptr<LaunchSlot[]> slots;
  u32 n_slots = 0;

  template <class T>
  int alloc(T** p, size_t count) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return report_cuda_error(e, "cudaMalloc (serving)");
    allocs.push_back(*p);
    return GPULDA_OK;
  }

  bool take(u64 n, u64* off) {  // first fit
    for (auto it = free_ext.begin(); it != free_ext.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        const u64 rest = it->second - n, o = it->first + n;
        free_ext.erase(it);
        if (rest) free_ext[o] = rest;
        pool_used += n;
        return true;
      }
    }
    return false;
  }
  u64 largest_free() const {
    u64 b = 0;
    for (auto& kv : free_ext) b = std::max(b, kv.second);
    return b;
  }
  void give(u64 off, u64 n) {
    pool_used -= n;
    auto it = free_ext.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_ext.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_ext.erase(nx);
    }
    if (it != free_ext.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_ext.erase(it);
      }
    }
  }
  // Pool words of a group of n requests with T tokens: words, topic scratch
  // and (launch mode) the descriptors.
  u64 extent_words(u64 n, u64 T) const {
    return 2 * align_up(std::max<u64>(T, 1), 64) + (persistent ? 0 : align_up(n * sizeof(FoldReq) / 4, 64));
  }

  ~Server() {
    if (persistent && ctl && copy_s) {  // stop the resident kernel
      static const u32 one = 1;
      cudaMemcpyAsync(ctl + 16, &one, 4, cudaMemcpyHostToDevice, copy_s);
      cudaStreamSynchronize(copy_s);
    }
    if (kern_s) cudaStreamSynchronize(kern_s);
    for (u32 i = 0; i < n_slots; ++i) {
      LaunchSlot& sl = slots[i];
      if (sl.s) cudaStreamSynchronize(sl.s);
      if (sl.done) cudaEventDestroy(sl.done);
      if (sl.s) cudaStreamDestroy(sl.s);
    }
    if (copy_s) cudaStreamSynchronize(copy_s);
    staging.reset();
    slots.reset();
    if (kern_ev) cudaEventDestroy(kern_ev);
    if (copy_s) cudaStreamDestroy(copy_s);
    if (kern_s) cudaStreamDestroy(kern_s);
    if (recs_host) cudaFreeHost(recs_host);
    for (void* p : allocs) cudaFree(p);
  }
};

int create_common(const GpuldaServeArgs* a, u32 K, u32 V, float alpha, std::unique_ptr<Server>& sv) {
  if (!a) return report_error(GPULDA_ERR_ARGS, "null GpuldaServeArgs");
  if (a->mode != GPULDA_SERVE_PERSISTENT && a->mode != GPULDA_SERVE_LAUNCH)
    return report_error(GPULDA_ERR_ARGS, "unknown serving mode");
  if (a->mode == GPULDA_SERVE_LAUNCH && (a->slots < 1 || a->slots > kMaxSlots))
    return report_error(GPULDA_ERR_ARGS, "launch mode: slots must be 1..64");
  if (a->mode == GPULDA_SERVE_PERSISTENT && a->slots > 32)
    return report_error(GPULDA_ERR_ARGS, "persistent mode: slots (request warps per SM) must be 0..32");
  if (K < 1 || V < 1 || !(alpha > 0.0f) || !std::isfinite(alpha))
    return report_error(GPULDA_ERR_ARGS, "model: K, V positive and alpha > 0");
  if (K > GPULDA_SERVE_MAX_K) return report_error(GPULDA_ERR_UNSUPPORTED, "K above GPULDA_SERVE_MAX_K");
  sv.reset(new Server());
  Server& s = *sv;
  s.K = K;
  s.V = V;
  s.alpha = alpha;
  s.args = *a;
  s.persistent = a->mode == GPULDA_SERVE_PERSISTENT;
  s.stage_cap = s.persistent ? kStagingBytes : kSlotStagingBytes;
  s.rec_bytes = record_bytes(K);
  s.max_inflight = a->max_inflight ? a->max_inflight : 16384u;
  const size_t cells = (size_t)K * V;
  FoldCommon& fc = s.fc;
  int rc;
  if ((rc = s.alloc(&fc.m.q, cells)) || (rc = s.alloc(&fc.m.al, cells)) || (rc = s.alloc(&fc.m.csr, cells)) ||
      (rc = s.alloc(&fc.m.A, V)) || (rc = s.alloc(&fc.m.nnz, V)) || (rc = s.alloc(&fc.status, 1)))
    return rc;
  fc.m.K = K;
  fc.m.V = V;
  fc.m.alpha = alpha;
  fc.rec_bytes = s.rec_bytes;
  fc.n_iter = a->n_iter;
  fc.key0 = (u32)a->seed;
  fc.key1 = a->chain;
  fc.n_recs = s.max_inflight;
  SCK(cudaMemset(fc.status, 0, 4));
  u64 pool = a->pool_bytes;
  if (!pool) {
    size_t fr = 0, tot = 0;
    SCK(cudaMemGetInfo(&fr, &tot));
    pool = std::min<u64>(fr / 2, 32ull << 30);
  }
  s.pool_words = pool / 4 / 64 * 64;
  if (!s.pool_words) return report_error(GPULDA_ERR_ARGS, "pool_bytes too small");
  if ((rc = s.alloc(&fc.pool, s.pool_words))) return rc;
  fc.pool_words = s.pool_words;
  s.free_ext[0] = s.pool_words;
  // result records: mapped pinned host memory, written by the kernels
  SCK(cudaHostAlloc((void**)&s.recs_host, (size_t)s.max_inflight * s.rec_bytes, cudaHostAllocMapped));
  SCK(cudaHostGetDevicePointer((void**)&fc.recs, s.recs_host, 0));
  s.free_recs.resize(s.max_inflight);
  for (u32 i = 0; i < s.max_inflight; ++i) s.free_recs[i] = s.max_inflight - 1 - i;
  const size_t smem = fold_smem_bytes(K);
  if (s.persistent) {
    s.resident_per_sm = a->slots ? a->slots : 32u;
    s.ring_cap = 1;
    while (s.ring_cap < 2ull * s.max_inflight) s.ring_cap <<= 1;
    if ((rc = s.alloc(&s.ring, s.ring_cap)) || (rc = s.alloc(&s.ctl, 64))) return rc;
    SCK(cudaMemset(s.ctl, 0, 64));
    SCK(cudaStreamCreateWithFlags(&s.copy_s, cudaStreamNonBlocking));
    SCK(cudaStreamCreateWithFlags(&s.kern_s, cudaStreamNonBlocking));
    SCK(cudaEventCreateWithFlags(&s.kern_ev, cudaEventDisableTiming));
    s.staging.reset(new Staging[kStaging]);
    for (u32 i = 0; i < kStaging; ++i)
      if ((rc = s.staging[i].init(kStagingBytes))) return rc;
    if (smem > 48 * 1024)
      SCK(cudaFuncSetAttribute(fold_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  } else {
    s.n_slots = a->slots;
    s.slots.reset(new LaunchSlot[a->slots]);
    for (u32 i = 0; i < s.n_slots; ++i) {
      LaunchSlot& sl = s.slots[i];
      SCK(cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking));
      SCK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
      if ((rc = sl.st.init(kSlotStagingBytes))) return rc;
    }
    if (smem > 48 * 1024)
      SCK(cudaFuncSetAttribute(fold_launch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  SCK(cudaDeviceSynchronize());
  return GPULDA_OK;
}

const unsigned char* rec_at(const Server& s, u32 rec) { return s.recs_host + (size_t)rec * s.rec_bytes; }

// Hands out every in-flight request whose done flag is up.
void collect(Server& s) {
  u64 t = 0;
  for (auto it = s.inflight.begin(); it != s.inflight.end();) {
    const unsigned char* rec = rec_at(s, it->rec);
    if (!__atomic_load_n((const u32*)(rec + ll_offset(s.K) + 12), __ATOMIC_ACQUIRE)) {
      ++it;
      continue;
    }
    if (!t) t = now_ns();
    Result res;
    res.id = it->id;
    res.theta.assign((const float*)rec, (const float*)rec + s.K);
    std::memcpy(&res.ll, rec + ll_offset(s.K), 8);
    std::memcpy(&res.skipped, rec + ll_offset(s.K) + 8, 4);
    res.done_ns = t;
    s.results.push_back(std::move(res));
    s.free_recs.push_back(it->rec);
    if (s.persistent) {  // a warp that raised the flag no longer reads the extent
      auto ex = s.extents.find(it->extent);
      if (ex != s.extents.end() && --ex->second.second == 0) {
        s.give(ex->first, ex->second.first);
        s.extents.erase(ex);
      }
    }
    ++s.finished;
    it = s.inflight.erase(it);
  }
}

// How many requests from the queue front fit the pool's largest free extent,
// a staging buffer, the free records and the cap; *T_out receives their
// token total.
u64 admissible(Server& s, u64 cap, u64* T_out) {
  const u64 room = s.largest_free();
  u64 n = 0, T = 0;
  const u64 lim = std::min<u64>(std::min<u64>(cap, (u64)s.free_recs.size()), (u64)s.queue.size());
  while (n < lim) {
    const u64 T2 = T + s.queue[n].words.size();
    if (s.extent_words(n + 1, T2) > room || staging_bytes(n + 1, T2) > s.stage_cap) break;
    T = T2;
    ++n;
  }
  if (!n && !s.queue.empty()) ++s.deferred;
  *T_out = T;
  return n;
}

// Moves the first n queued requests (T tokens) into the pool extent at off:
// their words go to staging at `words_at`, their descriptors to reqs (in
// launch order: longest first when asked), and they become in flight.
void stage(Server& s, u64 n, u64 T, u64 off, unsigned char* words_at, std::vector<FoldReq>& reqs,
           bool longest_first) {
  std::vector<u32> ord(n);
  for (u32 i = 0; i < n; ++i) ord[i] = i;
  if (longest_first)
    std::stable_sort(ord.begin(), ord.end(),
                     [&](u32 x, u32 y) { return s.queue[x].words.size() > s.queue[y].words.size(); });
  u32* wst = (u32*)words_at;
  const u64 zbase = off + align_up(std::max<u64>(T, 1), 64);
  reqs.resize(n);
  u64 tok = 0;
  for (u32 r = 0; r < n; ++r) {
    Req& q = s.queue[ord[r]];
    const u32 rec = s.free_recs.back();
    s.free_recs.pop_back();
    *(volatile u32*)(rec_at(s, rec) + ll_offset(s.K) + 12) = 0u;
    reqs[r] = FoldReq{off + tok, zbase + tok, q.id, (u32)q.words.size(), rec};
    if (!q.words.empty()) std::memcpy(wst + tok, q.words.data(), q.words.size() * 4);
    tok += q.words.size();
    s.inflight.push_back(InFlight{q.id, rec, off});
  }
  s.queue.erase(s.queue.begin(), s.queue.begin() + n);
}

int ensure_kernel(Server& s) {
  if (s.kern_live) {
    const cudaError_t e = cudaEventQuery(s.kern_ev);
    if (e == cudaErrorNotReady) return GPULDA_OK;
    if (e != cudaSuccess) return report_cuda_error(e, "persistent fold kernel");
    s.kern_live = false;
  }
  RingDev rd;
  rd.ring = s.ring;
  rd.cap = s.ring_cap;
  rd.head = (unsigned long long*)s.ctl;
  rd.tail = (const u64*)(s.ctl + 8);
  rd.stop = (const u32*)(s.ctl + 16);
  int fit = 0;
  SCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fold_persistent_kernel, 32, fold_smem_bytes(s.K)));
  const u32 blocks = (u32)device_sm_count() * std::max<u32>(1, std::min<u32>(s.resident_per_sm, (u32)fit));
  fold_persistent_kernel<<<blocks, 32, fold_smem_bytes(s.K), s.kern_s>>>(s.fc, rd);
  SCK(cudaGetLastError());
  SCK(cudaEventRecord(s.kern_ev, s.kern_s));
  s.kern_live = true;
  ++s.launches;
  return GPULDA_OK;
}

// Persistent mode: publishes admissible requests to the ring.
int publish(Server& s) {
  u64 T = 0;
  // every in-flight request holds at most one ring entry
  const u64 n = s.queue.empty() || s.published + s.queue.size() >= (1ull << 32)
                    ? 0
                    : admissible(s, s.ring_cap - s.inflight.size(), &T);
  if (n) {
    u64 off = 0;
    const u64 words = s.extent_words(n, T);
    if (!s.take(words, &off)) return report_error(GPULDA_ERR_NOMEM, "request pool");
    s.extents[off] = {words, (u32)n};
    Staging& st = s.staging[s.next_staging];
    s.next_staging = (s.next_staging + 1) % kStaging;
    // staging: [tail u64][pad][descriptors][words]
    const size_t head = staging_bytes(n, 0);
    int rc = st.ready();
    if (rc) return rc;
    std::vector<FoldReq> reqs;
    stage(s, n, T, off, st.p + head, reqs, false);
    std::memcpy(st.p + 16, reqs.data(), n * sizeof(FoldReq));
    const u64 new_tail = s.published + n;
    std::memcpy(st.p, &new_tail, 8);
    cudaStream_t cs = s.copy_s;
    if (T) SCK(cudaMemcpyAsync(s.fc.pool + off, st.p + head, T * 4, cudaMemcpyHostToDevice, cs));
    const u64 first = s.published & (s.ring_cap - 1);
    const u64 n1 = std::min<u64>(n, s.ring_cap - first);
    SCK(cudaMemcpyAsync(s.ring + first, st.p + 16, n1 * sizeof(FoldReq), cudaMemcpyHostToDevice, cs));
    if (n1 < n)
      SCK(cudaMemcpyAsync(s.ring, st.p + 16 + n1 * sizeof(FoldReq), (n - n1) * sizeof(FoldReq),
                          cudaMemcpyHostToDevice, cs));
    // The tail last: a warp that sees it finds the descriptors and words in
    // place.  Tails stay below 2^32, so a warp reading the 8-byte tail while
    // it is being written never sees a mix of old and new halves.
    SCK(cudaMemcpyAsync(s.ctl + 8, st.p, 8, cudaMemcpyHostToDevice, cs));
    SCK(cudaEventRecord(st.ev, cs));
    st.pending = true;
    s.published = new_tail;
  }
  // requests in flight need a live kernel (its warps leave when idle)
  return s.inflight.empty() ? GPULDA_OK : ensure_kernel(s);
}

// Launch mode: releases slots whose kernel finished, then launches batches.
int launch_batches(Server& s) {
  for (u32 i = 0; i < s.n_slots; ++i) {
    LaunchSlot& sl = s.slots[i];
    if (!sl.busy) continue;
    const cudaError_t e = cudaEventQuery(sl.done);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return report_cuda_error(e, "fold launch");
    s.give(sl.ext_off, sl.ext_words);
    sl.busy = false;
  }
  const u64 cap = s.args.max_batch ? s.args.max_batch : ~0ull;
  for (u32 i = 0; i < s.n_slots && !s.queue.empty(); ++i) {
    LaunchSlot& sl = s.slots[i];
    if (sl.busy) continue;
    u64 T = 0;
    const u64 n = admissible(s, cap, &T);
    if (!n) break;
    u64 off = 0;
    const u64 words = s.extent_words(n, T);
    if (!s.take(words, &off)) return report_error(GPULDA_ERR_NOMEM, "request pool");
    // staging: [header][descriptors][words]; pool extent: [words][topics][descriptors]
    const size_t head = staging_bytes(n, 0);
    std::vector<FoldReq> reqs;
    stage(s, n, T, off, sl.st.p + head, reqs, true);
    std::memcpy(sl.st.p + 16, reqs.data(), n * sizeof(FoldReq));
    u32* items = s.fc.pool + off + 2 * align_up(std::max<u64>(T, 1), 64);
    if (T) SCK(cudaMemcpyAsync(s.fc.pool + off, sl.st.p + head, T * 4, cudaMemcpyHostToDevice, sl.s));
    SCK(cudaMemcpyAsync(items, sl.st.p + 16, n * sizeof(FoldReq), cudaMemcpyHostToDevice, sl.s));
    fold_launch_kernel<<<(u32)n, 32, fold_smem_bytes(s.K), sl.s>>>(s.fc, (const FoldReq*)items);
    SCK(cudaGetLastError());
    SCK(cudaEventRecord(sl.done, sl.s));
    sl.busy = true;  // the staging buffer is reused once `done` has passed
    sl.ext_off = off;
    sl.ext_words = words;
    ++s.launches;
  }
  return GPULDA_OK;
}

int progress(Server& s) {
  collect(s);
  return s.persistent ? publish(s) : launch_batches(s);
}

bool idle(const Server& s) { return s.queue.empty() && s.inflight.empty(); }

Server* as_server(void* h) { return static_cast<Server*>(h); }

}  // namespace

extern "C" int gpulda_serve_create(const GpuldaServeArgs* args, void** handle) {
  if (!handle) return report_error(GPULDA_ERR_ARGS, "null handle pointer");
  *handle = nullptr;
  ModelDev src{};
  int t = -1;
  if (!current_model(&src, &t)) return report_error(GPULDA_ERR_STATE, "no initialized model to serve");
  if (t < 0) return report_error(GPULDA_ERR_STATE, "the model has no Phi yet (no sample_phi)");
  std::unique_ptr<Server> sv;
  int rc = create_common(args, src.K, src.V, src.alpha, sv);
  if (rc) return rc;
  Server& s = *sv;
  const size_t cells = (size_t)src.K * src.V;
  SCK(cudaMemcpy(s.fc.m.q, src.q, cells * 4, cudaMemcpyDeviceToDevice));
  SCK(cudaMemcpy(s.fc.m.al, src.al, cells * 8, cudaMemcpyDeviceToDevice));
  SCK(cudaMemcpy(s.fc.m.csr, src.csr, cells * 8, cudaMemcpyDeviceToDevice));
  SCK(cudaMemcpy(s.fc.m.A, src.A, (size_t)src.V * 8, cudaMemcpyDeviceToDevice));
  SCK(cudaMemcpy(s.fc.m.nnz, src.nnz, (size_t)src.V * 4, cudaMemcpyDeviceToDevice));
  SCK(cudaDeviceSynchronize());
  *handle = sv.release();
  return GPULDA_OK;
}

extern "C" int gpulda_serve_create_from_phi(const GpuldaServeArgs* args, uint32_t K, uint32_t V, float alpha,
                                            const uint32_t* q, void** handle) {
  if (!handle) return report_error(GPULDA_ERR_ARGS, "null handle pointer");
  *handle = nullptr;
  if (!q) return report_error(GPULDA_ERR_ARGS, "null Phi");
  std::unique_ptr<Server> sv;
  int rc = create_common(args, K, V, alpha, sv);
  if (rc) return rc;
  Server& s = *sv;
  const size_t cells = (size_t)K * V;
  SCK(cudaMemcpy(s.fc.m.q, q, cells * 4, cudaMemcpyHostToDevice));
  // The alias build turns raw draws x into floor(x * 2^32 / S); with S = 2^32
  // it keeps q as given and builds A, nnz, the nonzero lists and the alias
  // tables exactly as the Phi step does.
  std::vector<u64> ones(K, 1ull << 32);
  u64* S = nullptr;
  SCK(cudaMalloc(&S, (size_t)K * 8));
  cudaError_t e = cudaMemcpy(S, ones.data(), (size_t)K * 8, cudaMemcpyHostToDevice);
  void* scratch = nullptr;
  const size_t sb = alias_build_scratch_bytes(K);
  if (e == cudaSuccess && sb) e = cudaMalloc(&scratch, sb);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    ModelDev md = s.fc.m;
    md.S = S;
    md.Sinv = nullptr;  // a one-off build: plain divisions
    launch_alias_build(md, nullptr, scratch, sb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  cudaFree(S);
  if (scratch) cudaFree(scratch);
  if (e != cudaSuccess) return report_cuda_error(e, "serving model alias build");
  *handle = sv.release();
  return GPULDA_OK;
}

extern "C" int gpulda_serve_destroy(void* handle) {
  delete as_server(handle);
  return GPULDA_OK;
}

extern "C" int gpulda_serve_submit(void* handle, uint32_t n, const uint64_t* ids, const uint32_t* lengths,
                                   const uint32_t* words) {
  Server* s = as_server(handle);
  if (!s) return report_error(GPULDA_ERR_ARGS, "null serving handle");
  if (n && (!ids || !lengths)) return report_error(GPULDA_ERR_ARGS, "null request arrays");
  u64 total = 0;
  for (u32 r = 0; r < n; ++r) {
    if (lengths[r] > GPULDA_MAX_DOC_LEN) return report_error(GPULDA_ERR_UNSUPPORTED, "request above GPULDA_MAX_DOC_LEN");
    if (s->extent_words(1, lengths[r]) > s->pool_words)
      return report_error(GPULDA_ERR_UNSUPPORTED, "request larger than the request pool");
    total += lengths[r];
  }
  if (total && !words) return report_error(GPULDA_ERR_ARGS, "null words");
  for (u64 i = 0; i < total; ++i)
    if (words[i] >= s->V) return report_error(GPULDA_ERR_ARGS, "word id >= V");
  u64 pos = 0;
  for (u32 r = 0; r < n; ++r) {
    Req q;
    q.id = ids[r];
    q.words.assign(words + pos, words + pos + lengths[r]);
    pos += lengths[r];
    s->queue.push_back(std::move(q));
  }
  return GPULDA_OK;
}

extern "C" int gpulda_serve_progress(void* handle) {
  Server* s = as_server(handle);
  if (!s) return report_error(GPULDA_ERR_ARGS, "null serving handle");
  return progress(*s);
}

extern "C" int gpulda_serve_poll(void* handle, uint32_t max, uint64_t* ids, float* theta, double* loglik,
                                 uint32_t* skipped, uint64_t* done_ns, uint32_t* n_out) {
  Server* s = as_server(handle);
  if (!s || !ids || !n_out) return report_error(GPULDA_ERR_ARGS, "bad serve_poll arguments");
  u32 n = 0;
  while (n < max && !s->results.empty()) {
    Result& r = s->results.front();
    ids[n] = r.id;
    if (theta) std::memcpy(theta + (size_t)n * s->K, r.theta.data(), (size_t)s->K * 4);
    if (loglik) loglik[n] = r.ll;
    if (skipped) skipped[n] = r.skipped;
    if (done_ns) done_ns[n] = r.done_ns;
    s->results.pop_front();
    ++n;
  }
  *n_out = n;
  return GPULDA_OK;
}

extern "C" int gpulda_serve_drain(void* handle) {
  Server* s = as_server(handle);
  if (!s) return report_error(GPULDA_ERR_ARGS, "null serving handle");
  u64 last_change = now_ns();
  u64 seen = s->finished;
  while (!idle(*s)) {
    const int rc = progress(*s);
    if (rc) return rc;
    if (s->finished != seen) {
      seen = s->finished;
      last_change = now_ns();
    } else if (now_ns() - last_change > kDrainStallNs) {
      return report_error(GPULDA_ERR_STATE, "drain: no request finished for 120 s");
    } else {
      timespec ts{0, 20000};  // 20 us
      nanosleep(&ts, nullptr);
    }
  }
  // launch mode: wait for the slots (their extents are released then)
  if (!s->persistent) {
    for (u32 i = 0; i < s->n_slots; ++i)
      if (s->slots[i].busy) SCK(cudaEventSynchronize(s->slots[i].done));
    const int rc = launch_batches(*s);
    if (rc) return rc;
  }
  u32 st = 0;
  SCK(cudaMemcpy(&st, s->fc.status, 4, cudaMemcpyDeviceToHost));
  if (st) {
    SCK(cudaMemset(s->fc.status, 0, 4));
    return report_error(GPULDA_ERR_DEVICE, "fold-in: device status set");
  }
  return GPULDA_OK;
}

extern "C" int gpulda_serve_stats(void* handle, uint64_t* out, int n) {
  Server* s = as_server(handle);
  if (!s || !out) return 0;
  const uint64_t v[10] = {s->queue.size(), s->inflight.size(), s->results.size(), s->launches, s->finished,
                          s->pool_words * 4, s->pool_used * 4, s->deferred, s->K, s->V};
  const int m = n < 10 ? n : 10;
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}
