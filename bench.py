"""Gibbs-sweep benchmark of libGPUPolyaUrnLDA.so (one JSON line on rank 0).

A step is one full Gibbs iteration over the whole corpus: the Phi step
(Poisson draws, normalisers, alias tables) and one z sweep that resamples
every token and rebuilds the counts.  Default workload: the mid configuration
(K=1000, V=100000, D=300000, ~1.0e8 tokens; synthetic, seeded).

  value   tokens/s with the corpus resident in HBM (gpulda_corpus_sweep),
          device time from CUDA events on the library's stream, max over ranks
  e2e     tokens/s through the reference protocol (initialize / sample_phi /
          sample_z_async / sync_buffer) with pinned host buffers: every step
          copies z, w, d, K_d to the device and z back
  roofline  the z-sweep kernel's algorithmic bytes (24 N + 8 D + 4 S, S the
          sparse work counted by the kernel) over its CUDA-event time,
          against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (same algorithm) on a bounded sample, all cores
  serving  fold-in requests against the trained model at 1k and 50k docs/s
          offered: continuous batching vs one launch per document

--impl reference times the CPU oracle alone (the reference has no CPU
implementation of the path, and its CUDA kernels do not build for sm_100a).
Multi-GPU (torchrun): independent chains per GPU (replicas), weak scaling;
--shard: one chain with its documents sharded across the GPUs.
Other workloads: --workload batched (64 independent problems in one graph),
--workload serve (the serving comparison at several rates), large_k1000,
large_k10000.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "gibbs_tokens_per_sec"
UNIT = "tokens/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="mid")
    p.add_argument("--docs", type=int, default=None, help="override the number of documents")
    p.add_argument("--vocab", type=int, default=None,
                   help="override the vocabulary size (small profiling cases of the large-K workloads)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-serve", action="store_true", help="skip the serving summary of the default line")
    p.add_argument("--no-large", action="store_true", help="skip the large-K summary of the default line")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-chains summary of the default line")
    p.add_argument("--large-steps", type=int, default=3, help="large-K summary: timed iterations")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU seconds per timed oracle iteration")
    p.add_argument("--problems", type=int, default=64, help="batched workload: number of problems")
    p.add_argument("--batch-scale", type=float, default=1.0, help="batched workload: scale of each problem's D")
    p.add_argument("--tune-cache", default=None, help="batched workload: autotuner cache file")
    p.add_argument("--rates", type=int, nargs="+", default=[1000, 10000, 50000], help="serve: offered docs/s")
    p.add_argument("--serve-requests", type=int, default=100000, help="serve: max requests per rate")
    p.add_argument("--serve-seconds", type=float, default=2.0, help="serve: seconds of arrivals per rate")
    p.add_argument("--serve-unbatched", type=int, default=3000, help="serve: requests of the unbatched run")
    p.add_argument("--serve-train", type=int, default=5, help="serve: training iterations of the model")
    p.add_argument("--serve-slots", type=int, default=32, help="serve: launches in flight")
    p.add_argument("--shard", action="store_true",
                   help="one chain with its documents sharded across the ranks (strong scaling; default: replicas)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every 50 ms) during the timed region: start() returns
    once the first sample has arrived, and stop() keeps the samples taken
    between the two calls."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 5.0
            while not self.rows and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.monotonic(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t1 = time.monotonic()
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        rows = [r for t, r in self.rows if self.t0 <= t <= t1] or [r for _, r in self.rows[-1:]]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, device) -> float:
    """Max of a per-rank timing over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_tokens: int, steps: int, world: int, seconds_max: float) -> float:
    """Whole-job tokens/s of `world` independent chains (one per GPU, each over
    the full corpus): every rank sweeps n_tokens per step; the job takes the
    slowest rank's time."""
    return world * n_tokens * steps / seconds_max


def measured_traffic_per_token():
    """DRAM bytes per token of the z-sweep kernel from the committed ncu
    summary (a smaller case of the same workload; traffic scales with tokens)."""
    try:
        with open(os.path.join(ROOT, "profiles", "z_sweep_kernel_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_token"])
    except Exception:
        return None


def roofline_profile(workload: str, c) -> dict:
    """The roofline keys that come from the committed ncu profile: it covers
    the dense-count z sweep on a slice of the mid workload, so its traffic is
    scaled to this launch only for that workload."""
    if c.K > 2048:
        return {"kernel": "z_sweep_pairs_kernel", "traffic": None,
                "traffic_note": "the committed ncu capture of this kernel is a V=14,000 case "
                                "(profiles/z_sweep_pairs_kernel_K10000_small_case.md: about 1.2 kB of DRAM traffic per "
                                "token at a 49 % L2 hit rate); its hit rate does not carry over to V=140,000, so no "
                                "traffic is scaled to this launch"}
    out = {"kernel": "z_sweep_kernel",
           "binding_resource": "L1 data pipe (74 % of wavefront slots in the ncu profile), issue (66 %) and "
                               "gather latency; DRAM at 2.6 %: 93 % of the gathers hit L2, half of them L1"}
    tpt = measured_traffic_per_token()
    if workload == "mid" and tpt:
        out.update(traffic=tpt * c.n_tokens, traffic_note="ncu dram bytes per token of a 3.4e7-token slice, scaled to N")
    else:
        out.update(traffic=None, traffic_note="the committed ncu capture covers the mid workload only")
    return out


def make_corpus(args, device):
    import dataclasses
    from gpupolyaurnlda_b200 import corpus
    wl = corpus.WORKLOADS[args.workload]
    if getattr(args, "vocab", None):
        wl = dataclasses.replace(wl, V=args.vocab)
    return corpus.generate(wl, seed=1, device=device, D=args.docs)


def workload_desc(c, args):
    return {"workload": f"{args.workload}: K={c.K} V={c.V} D={c.n_docs} N={c.n_tokens} tokens "
                        f"(synthetic LDA corpus, seed 1; random initial topics)",
            "K": c.K, "V": c.V, "D": c.n_docs, "N": c.n_tokens, "alpha": c.alpha, "beta": c.beta,
            "l2": "inputs larger than L2 (fixed-point Phi 4KV B, alias tables 8KV B, corpus 8N B)"}


class CpuChain:
    """The CPU oracle's sweep (same algorithm and random streams) on a leading
    slice of the documents, sized so one iteration takes about `seconds`.
    Each step is one full iteration of that chain: the Phi step over all K*V
    cells and a z sweep over the slice; tokens/s is extrapolated to the whole
    corpus as N / (t_phi + t_z * N / n_slice)."""

    def __init__(self, c, seconds: float, threads: int | None = None):
        import oracle
        self.lib_path = oracle_native(oracle)
        self.c = c
        self.threads = threads or oracle.default_threads()
        self.ch = oracle.Chain(c.K, c.alpha, c.beta, c.counts, seed=0, threads=self.threads)
        cum = np.cumsum(c.d_len.astype(np.int64))
        # probe: one Phi step and a sweep of ~2e5 tokens
        t0 = time.perf_counter()
        self.ch.sample_phi()
        t_phi = time.perf_counter() - t0
        pd = min(c.n_docs, int(np.searchsorted(cum, min(c.n_tokens, 200000))) + 1)
        pt = int(cum[pd - 1])
        t0 = time.perf_counter()
        self.ch.sweep(c.w[:pt], c.z[:pt].copy(), c.d_len[:pd])
        rate = pt / max(1e-9, time.perf_counter() - t0)
        want = int(min(c.n_tokens, max(pt, rate * max(1.0, seconds - t_phi))))
        self.docs = min(c.n_docs, int(np.searchsorted(cum, want)) + 1)
        self.ntok = int(cum[self.docs - 1])
        self.z = c.z[:self.ntok].copy()
        self.ch = oracle.Chain(c.K, c.alpha, c.beta, c.counts, seed=0, threads=self.threads)
        self.last = None

    def step(self) -> float:
        t0 = time.perf_counter()
        self.ch.sample_phi()
        t_phi = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.ch.sweep(self.c.w[:self.ntok], self.z, self.c.d_len[:self.docs])
        t_z = time.perf_counter() - t0
        self.last = (t_phi, t_z)
        return self.c.n_tokens / (t_phi + t_z * (self.c.n_tokens / self.ntok))

    def describe(self, value: float, warm: int) -> dict:
        t_phi, t_z = self.last
        return {"value": value, "unit": UNIT, "cores": self.threads, "kind": "port", "build": self.lib_path,
                "sample": f"CPU oracle chain on the first {self.docs} documents ({self.ntok} of {self.c.n_tokens} "
                          f"tokens) after {warm} warm-up iterations; per iteration a Phi step over all "
                          f"{self.c.K}x{self.c.V} cells ({t_phi:.2f} s) and a z sweep of the slice ({t_z:.2f} s), "
                          f"extrapolated to the whole corpus"}


def oracle_native(oracle) -> str:
    """The timed CPU legs run the oracle built with -march=native on this host
    (oracle/build.py; same results bit for bit as the portable build)."""
    if oracle._lib is None:
        oracle.use_native_build()
    return os.path.basename(oracle._path)


def cpu_baseline(c, seconds: float, warm: int = 2):
    cc = CpuChain(c, seconds)
    for _ in range(warm):
        cc.step()
    v = cc.step()
    return cc.describe(v, warm)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    dev = "cuda" if _cuda() else "cpu"
    c = make_corpus(args, dev)
    cc = CpuChain(c, args.cpu_seconds)
    vals = []
    for i in range(args.warmup + args.steps):
        v = cc.step()
        if i >= args.warmup:
            vals.append(v)
    v = float(np.median(vals))
    ms = c.n_tokens / v * 1e3
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "impl": "reference",
            "config": workload_desc(c, args), "parallelism": f"CPU, {cc.threads} threads",
            "cpu_baseline": cc.describe(v, args.warmup),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU oracle port of the sweep (the reference has no CPU implementation of the path; its CUDA "
                    "kernels are not run on this pool)"}
    print(json.dumps(line), flush=True)


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def run_ours(args):
    import torch
    import torch.distributed as dist

    import gpupolyaurnlda_b200 as g

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    c = make_corpus(args, f"cuda:{local}")
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()  # the library's work and the timing events share it
    hbm, peak_kind = peaks()

    # ---- device-resident corpus: value + roofline ----------------------------
    s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=0, chain=rank)
    s.set_stream(stream.cuda_stream)
    s.corpus_load(c.z.copy(), c.w, c.d_len)
    for _ in range(args.warmup):
        s.corpus_sweep(1)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    z_ms, phi_ms, S_work, launches = [], [], [], 0
    draw_ms, alias_ms = [], []
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        s.corpus_sweep(1)  # host-synchronous; events below bracket all steps
        kt = s.kernel_times()
        cnt = s.counters()
        z_ms.append(kt["z_sweep"])
        phi_ms.append(kt["phi_draw"] + kt["alias_build"] + kt["prep"])
        draw_ms.append(kt["phi_draw"])
        alias_ms.append(kt["alias_build"])
        S_work.append(cnt["sparse_work"])
        launches += cnt["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_max = max_over_ranks(e0.elapsed_time(e1), f"cuda:{local}")
    if world > 1:
        dist.barrier()
    s.set_stream(0)
    nnz_total = int(s.read_state(n=False, q=False, alias=False, A=False, S=False)["nnz"].astype(np.int64).sum())
    # the standalone count rebuild over the same topics (leaves n as the last sweep rebuilt it)
    rebuild_ms = float(np.median([s.corpus_count_rebuild() for _ in range(3)]))

    # ---- serving fold-in against the model just trained (one GPU) ----------
    serving = None
    if world == 1 and not args.no_serve and c.K <= 2048:
        from gpupolyaurnlda_b200.serve import Server
        srv_b = Server(50, seed=0, max_inflight=1 << 17)
        srv_u = Server(50, mode="launch", slots=args.serve_slots, max_batch=1, seed=0)
        q_model = s.read_state(n=False, alias=False, A=False, S=False, nnz=False)["q"]
        s.close()
        rows, ll = serve_measure(srv_b, srv_u, q_model, [1000, 10000, 50000], 2.0, 100000, 3000, local)
        srv_b.close()
        srv_u.close()
        serving = {"metric": "served_docs_per_sec", "unit": "docs/s",
                   "workload": f"the chain's model after {args.warmup + args.steps} iterations, {SERVE_WORKLOAD}; "
                               f"batched = persistent kernel (32 request warps per SM), unbatched = one launch per "
                               f"document over {args.serve_slots} streams",
                   "rates": [{"offered": r["offered_docs_per_sec"], "requests": r["requests"],
                              "batched": r["batched"], "unbatched": r["unbatched"],
                              "speedup": r["batched"]["docs_per_sec"] / r["unbatched"]["docs_per_sec"],
                              "results_identical": r["results_identical"]} for r in rows],
                   "heldout_ll_per_token": ll}
    else:
        s.close()

    large = batched = None
    if world == 1 and not args.no_large and args.workload == "mid":
        large = large_k_measure(args, local, hbm)
    if world == 1 and not args.no_batched and args.workload == "mid":
        import argparse as _ap
        bargs = _ap.Namespace(**vars(args))
        bargs.steps, bargs.warmup = 3, 2
        r = batched_measure(bargs, local, 1, 0)
        batched = {k: r[k] for k in ("value", "ms_per_step", "steps", "warmup", "workload", "mode", "sequential",
                                     "speedup_vs_sequential", "loglik_max_rel_diff_vs_solo", "autotuner", "clocks")}
        batched["metric"] = "batched_gibbs_tokens_per_sec"
        torch.cuda.empty_cache()

    value = replica_value(c.n_tokens, args.steps, world, ms_max / 1e3)
    zb = [24 * c.n_tokens + 8 * c.n_docs + 4 * S for S in S_work]
    z_gbs = float(np.mean([b / (m / 1e3) / 1e9 for b, m in zip(zb, z_ms)]))
    B_iter = [20 * c.K * c.V + b for b in zb]
    it_gbs = float(np.mean([b / (ms_max / args.steps / 1e3) / 1e9 for b in B_iter]))

    # ---- reference protocol through the C ABI: e2e ---------------------------
    # Pinned host buffers (gpulda_pin_host exists for callers that can pin),
    # and pageable ones: the reference's host maps its files pageable
    # (src/train.rs:77-83), the default path of a caller that does nothing more.
    e2e = e2e_pageable = None
    if not args.no_e2e:
        def protocol(zn, wn, dn, kn):
            s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=c.n_tokens, max_D=c.n_docs, seed=0,
                          chain=rank)
            for _ in range(args.warmup):
                s.sample_phi()
                s.sweep_buffer(0, zn, wn, dn, kn)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                s.sample_phi()
                s.sweep_buffer(0, zn, wn, dn, kn)
            el = max_over_ranks(time.perf_counter() - t0, f"cuda:{local}")
            s.close()
            return {"value": replica_value(c.n_tokens, args.steps, world, el), "unit": UNIT,
                    "h2d_bytes_per_step": 8 * c.n_tokens + 8 * c.n_docs, "d2h_bytes_per_step": 4 * c.n_tokens}

        zp = torch.from_numpy(c.z.copy()).pin_memory()
        wp = torch.from_numpy(c.w).pin_memory()
        dp = torch.from_numpy(c.d_len).pin_memory()
        kp = torch.from_numpy(c.k_d()).pin_memory()
        e2e = dict(protocol(zp.numpy(), wp.numpy(), dp.numpy(), kp.numpy()),
                   path="initialize/sample_phi/sample_z_async/sync_buffer, one buffer per iteration, pinned host")
        del zp, wp, dp, kp
        e2e_pageable = dict(protocol(c.z.copy(), c.w, c.d_len, c.k_d()),
                            path="the same protocol with pageable host arrays (no pinning)")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(c, args.cpu_seconds / 3, warm=2)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": workload_desc(c, args),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "roofline": dict({"bound": "hbm", "achieved": z_gbs, "peak": hbm, "unit": "GB/s",
                                  "frac": z_gbs / hbm,
                                  "algorithmic_bytes_per_launch": float(np.mean(zb)), "peak_kind": peak_kind},
                                 **roofline_profile(args.workload, c)),
                "iteration_roofline": {"achieved": it_gbs, "frac": it_gbs / hbm,
                                       "bytes_per_iteration": float(np.mean(B_iter))},
                "kernel_ms": {"z_sweep": float(np.mean(z_ms)), "phi_step": float(np.mean(phi_ms))},
                "kernel_gbs": {
                    "note": "algorithmic bytes / CUDA-event time per kernel: Poisson draw 12 B per (word, topic) "
                            "cell (read n, write x, zero n); alias build 8 B per cell + 16 B per nonzero Phi "
                            "(list and alias entry); z sweep as in roofline (the count rebuild is its atomics)",
                    "phi_draw": 12 * c.K * c.V / (float(np.mean(draw_ms)) / 1e3) / 1e9,
                    "alias_build": (8 * c.K * c.V + 16 * nnz_total) / (float(np.mean(alias_ms)) / 1e3) / 1e9,
                    "z_sweep": z_gbs,
                    "count_rebuild": 16 * c.n_tokens / (rebuild_ms / 1e3) / 1e9,
                    "count_rebuild_note": "gpulda_corpus_count_rebuild over the corpus's topics after the timed "
                                          "iterations: 16 B per token (read w and z, read-modify-write n), "
                                          "warp-aggregated atomics; the sweep fuses the same rebuild"},
                "sparse_work_per_token": float(np.mean(S_work)) / c.n_tokens,
                "gpu_launches": launches, "clocks": clk, "e2e": e2e, "e2e_pageable": e2e_pageable,
                "cpu_baseline": cpu, "serving": serving, "large_k10000": large, "batched": batched}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def large_k_measure(args, local: int, hbm: float, workload: str = "large_k10000") -> dict:
    """The large sweep at K=10000 (V=140,000, D=8,000,000, ~6.4e8 tokens;
    the sorted-pair-list store) with the corpus resident: 2 warm-up iterations,
    then `args.large_steps` timed ones (CUDA events on the library's stream).
    A summary beside the headline, not a second headline."""
    import torch

    import gpupolyaurnlda_b200 as g
    from gpupolyaurnlda_b200 import corpus
    t0 = time.perf_counter()
    c = corpus.generate(workload, seed=1, device=f"cuda:{local}")
    t_gen = time.perf_counter() - t0
    torch.cuda.empty_cache()  # the generator's buffers
    stream = torch.cuda.Stream()
    s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=0)
    s.set_stream(stream.cuda_stream)
    s.corpus_load(c.z.copy(), c.w, c.d_len)
    s.corpus_sweep(2)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    z_ms, phi_ms, S_work = [], [], []
    e0.record(stream)
    for _ in range(args.large_steps):
        s.corpus_sweep(1)
        kt = s.kernel_times()
        z_ms.append(kt["z_sweep"])
        phi_ms.append(kt["phi_draw"] + kt["alias_build"] + kt["prep"])
        S_work.append(s.counters()["sparse_work"])
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.large_steps
    s.set_stream(0)
    s.close()
    zb = [24 * c.n_tokens + 8 * c.n_docs + 4 * S for S in S_work]
    z_gbs = float(np.mean([b / (m / 1e3) / 1e9 for b, m in zip(zb, z_ms)]))
    out = {"workload": f"{workload}: K={c.K} V={c.V} D={c.n_docs} N={c.n_tokens} (synthetic, seed 1), iterations "
                       f"3..{2 + args.large_steps} of a chain from random topics",
           "tokens_per_s": c.n_tokens / (ms / 1e3), "ms_per_iteration": ms,
           "z_sweep_ms": float(np.mean(z_ms)), "phi_step_ms": float(np.mean(phi_ms)),
           "z_kernel": "z_sweep_pairs_kernel (sorted (topic, count) lists)",
           "roofline_frac": z_gbs / hbm, "z_achieved_gbs": z_gbs,
           "sparse_work_per_token": float(np.mean(S_work)) / c.n_tokens, "generate_s": t_gen, "clocks": clk}
    del c
    return out


def batched_problems(args, device, chain: int):
    """The batched-chains workload (corpus.batched_workloads): problem i drawn
    with data seed 1000 + i, sampled with seed i and the given chain."""
    from gpupolyaurnlda_b200 import corpus
    from gpupolyaurnlda_b200.batch import ProblemSpec
    specs = []
    for i, wl in enumerate(corpus.batched_workloads(args.problems, seed=1, D_scale=args.batch_scale)):
        c = corpus.generate(wl, seed=1000 + i, device=device)
        specs.append(ProblemSpec(c.alpha, c.beta, c.K, c.counts, c.z, c.w, c.d_len, seed=i, chain=chain))
    return specs


BATCH_MODES = {0: "per-bucket concurrent branches",
               1: "merged: one launch per stage over every problem",
               2: "merged sweep: per-bucket Phi-step branches, one z sweep over every problem's documents"}


def batched_measure(args, local: int, world: int, rank: int) -> dict:
    """Batched chains: all problems in one graph-replayed iteration (after the
    autotuner), against the same problems run one after another as solo
    models (the same iterations, seeds and chains, so the final
    log-likelihoods must agree).  Returns the measurement."""
    import torch

    import gpupolyaurnlda_b200 as g
    from gpupolyaurnlda_b200.batch import BatchChains

    t0 = time.perf_counter()
    specs = batched_problems(args, f"cuda:{local}", rank)
    t_gen = time.perf_counter() - t0
    N = sum(len(sp.z) for sp in specs)
    D = sum(len(sp.d_len) for sp in specs)
    stream = torch.cuda.Stream()  # graph launches and timing events share it
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    t0 = time.perf_counter()
    b = BatchChains(specs)
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    n_tuned = b.tune(args.tune_cache)
    t_tune = time.perf_counter() - t0
    shapes = b.shapes()
    info = b.info()
    b.sweep_async(args.warmup, stream.cuda_stream)
    b.sync()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    b.sweep_async(args.steps, stream.cuda_stream)
    e1.record(stream)
    b.sync()
    clk = clocks.stop()
    ms_max = max_over_ranks(e0.elapsed_time(e1), f"cuda:{local}")
    ll_b, _ = b.loglik()
    b.close()

    # the same problems one after another, each a solo model
    seq_ms, ll_s = 0.0, []
    for sp in specs:
        s = g.Sampler(sp.alpha, sp.beta, sp.K, sp.counts, buffer_size=16, max_D=4, seed=sp.seed, chain=sp.chain,
                      flags=g.GPULDA_FLAG_LOGLIK)
        s.set_stream(stream.cuda_stream)
        s.corpus_load(sp.z.copy(), sp.w, sp.d_len)
        s.corpus_sweep(args.warmup)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            s.corpus_sweep(1)
        e1.record(stream)
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        ll_s.append(s.loglik()[0])
        s.set_stream(0)
        s.close()
    seq_max = max_over_ranks(seq_ms, f"cuda:{local}")
    rel = max(abs(a - c) / abs(c) for a, c in zip(ll_b, ll_s))
    value = replica_value(N, args.steps, world, ms_max / 1e3)
    seq_value = replica_value(N, args.steps, world, seq_max / 1e3)
    Ks = [sp.K for sp in specs]
    return {"value": value, "ms_per_step": ms_max / args.steps, "steps": args.steps, "warmup": args.warmup,
            "workload": f"batched: {len(specs)} independent problems, K in {{50,200,1000}} "
                        f"({Ks.count(50)}/{Ks.count(200)}/{Ks.count(1000)}), V in [5k,50k], "
                        f"D in [1k,100k] x{args.batch_scale}, doc lengths lognormal(4.5,1.0); "
                        f"N={N} tokens, D={D} documents",
            "N": N, "D": D, "cells": info["cells"], "device_bytes": info["device_bytes"],
            "mode": BATCH_MODES.get(info.get("mode"), "?"),
            "sequential": {"value": seq_value, "unit": UNIT, "ms_per_step": seq_max / args.steps,
                           "what": "the same problems one after another as solo models (gpulda_corpus_sweep), "
                                   "device time summed"},
            "speedup_vs_sequential": value / seq_value,
            "loglik_max_rel_diff_vs_solo": rel,
            "autotuner": {"entries_tuned": n_tuned, "seconds": t_tune,
                          "shapes": {b_: list(sh) for b_, sh in zip(("K<=64", "K<=256", "K<=1024", "K<=2048"),
                                                                     shapes) if sh[0]}},
            "setup_seconds": {"generate": t_gen, "create": t_create},
            "gpu_launches": args.steps * (1 + {1: 3, 2: 2 * info["buckets"] + 1}.get(info.get("mode"), 3 * info["buckets"])),
            "clocks": clk}


def run_batched(args):
    """The batched-chains workload as its own line."""
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    r = batched_measure(args, local, world, rank)
    if rank == 0:
        line = {"metric": "batched_gibbs_tokens_per_sec", "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic",
                "config": {"workload": r["workload"], "N": r["N"], "D": r["D"], "cells": r["cells"],
                           "device_bytes": r["device_bytes"], "l2": "inputs larger than L2"},
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
        line.update({k: r[k] for k in ("mode", "sequential", "speedup_vs_sequential", "loglik_max_rel_diff_vs_solo",
                                       "autotuner", "setup_seconds", "gpu_launches", "clocks")})
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def serve_open_loop(srv, lengths, words, arrival_s, ids, keep_theta: int = 0):
    """Submits requests at their arrival times (open loop), keeps the server
    progressing and collects results.  Returns docs/s (requests over the time
    from the first arrival to the last completion), latencies (ns, completion
    minus scheduled arrival), per-request log-likelihoods and skipped counts
    in request order, and the theta rows of the first `keep_theta` requests."""
    n = len(lengths)
    K = srv.K
    offs = np.concatenate([[0], np.cumsum(lengths.astype(np.int64))])
    t0 = time.monotonic_ns() + 2_000_000
    arr = t0 + (arrival_s * 1e9).astype(np.int64)
    lat = np.zeros(n, np.int64)
    ll = np.zeros(n, np.float64)
    sk = np.zeros(n, np.int64)
    theta = np.zeros((keep_theta, K), np.float32)
    seen = np.zeros(n, bool)
    i = done = 0
    last = 0
    while done < n:
        now = time.monotonic_ns()
        j = int(np.searchsorted(arr, now, side="right"))
        busy = False
        if j > i:
            srv.submit(ids[i:j], lengths[i:j], words[offs[i]:offs[j]])
            i = j
            busy = True
        srv.progress()
        out = srv.poll(1 << 14, theta=keep_theta > 0)
        k = len(out["ids"])
        if k:
            r = (out["ids"] - ids[0]).astype(np.int64)
            lat[r] = out["done_ns"].astype(np.int64) - arr[r]
            ll[r] = out["ll"]
            sk[r] = out["skipped"]
            seen[r] = True
            if keep_theta:
                m = r < keep_theta
                theta[r[m]] = out["theta"][m]
            last = max(last, int(out["done_ns"].max()))
            done += k
            busy = True
        if not busy:
            time.sleep(2e-5)
    assert seen.all()
    return n / ((last - arr[0]) / 1e9), lat, ll, sk, theta


def serve_measure(srv_b, srv_u, q, rates, seconds, max_requests, max_unbatched, local):
    """Open-loop serving runs at the given offered rates against the batched
    (persistent) and the one-launch-per-document servers.  Requests are
    documents drawn from the served model's own topics (model_requests); each
    server folds in the first half of every document, and the second halves
    are scored by document completion (completion_loglik) with the theta each
    server returned, on the requests both servers ran.  Returns the per-rate
    rows and the held-out log-likelihood per token of both servers, beside
    that of a uniform theta."""
    from gpupolyaurnlda_b200.serve import completion_loglik, model_requests, split_halves
    K = srv_b.K
    rows = []
    acc = {"batched": [0.0, 0], "unbatched": [0.0, 0], "uniform theta": [0.0, 0]}
    for rate in rates:
        n = int(min(max(seconds * rate, 2000), max_requests))
        full_len, full_words = model_requests(q, K, n, seed=rate, device=f"cuda:{local}")
        lengths, words, h_len, h_words = split_halves(full_len, full_words)
        rng = np.random.default_rng(rate + 1)
        arrival = np.cumsum(rng.exponential(1.0 / rate, n))
        ids = np.arange(n, dtype=np.uint64) + np.uint64(rate) * np.uint64(1 << 32)
        nu = min(n, max_unbatched)
        clocks = ClockSampler(local)
        clocks.start()
        dps_b, lat_b, ll_b, sk_b, th_b = serve_open_loop(srv_b, lengths, words, arrival, ids, keep_theta=nu)
        clk = clocks.stop()
        dps_u, lat_u, ll_u, sk_u, th_u = serve_open_loop(srv_u, lengths[:nu], words[:int(lengths[:nu].sum())],
                                                         arrival[:nu], ids[:nu], keep_theta=nu)
        same = bool((ll_b[:nu] == ll_u).all() and (sk_b[:nu] == sk_u).all() and
                    (th_b.view(np.uint32) == th_u.view(np.uint32)).all())
        hw = h_words[:int(h_len[:nu].astype(np.int64).sum())]
        for name, th in (("batched", th_b), ("unbatched", th_u), ("uniform theta", np.full_like(th_b, 1.0 / K))):
            tot, cnt = completion_loglik(q, K, th, h_len[:nu], hw, device=f"cuda:{local}")
            acc[name][0] += tot
            acc[name][1] += cnt
        rows.append({"offered_docs_per_sec": rate, "requests": n, "tokens_folded_in": int(lengths.sum()),
                     "batched": {"docs_per_sec": dps_b, "p50_ms": float(np.percentile(lat_b, 50) / 1e6),
                                 "p99_ms": float(np.percentile(lat_b, 99) / 1e6)},
                     "unbatched": {"requests": nu, "docs_per_sec": dps_u,
                                   "p50_ms": float(np.percentile(lat_u, 50) / 1e6),
                                   "p99_ms": float(np.percentile(lat_u, 99) / 1e6)},
                     "results_identical": same, "clocks": clk})
    ll = {k: v[0] / max(1, v[1]) for k, v in acc.items()}
    ll["rel_diff"] = abs(ll["batched"] - ll["unbatched"]) / abs(ll["unbatched"])
    ll["tokens_scored"] = acc["batched"][1]
    ll["definition"] = ("document completion: fold in the first ceil(L/2) tokens (50 iterations, Phi fixed), "
                        "score the rest by log sum_k theta_k Phi[k][w] per token")
    return rows, ll


SERVE_WORKLOAD = ("documents drawn from the served model's topics (theta ~ Dir(0.1)), lengths lognormal(5.0,1.2) "
                  "clipped [5,20000], the first half of each folded in with 50 iterations, Poisson arrivals")


def run_serve(args):
    """Serving fold-in: a K=1000, V=100000 model trained on the mid corpus is
    served to Poisson arrivals of Zipf documents (lengths lognormal(5.0, 1.2)
    clipped to [5, 20000]), 50 fold-in iterations each; continuous batching
    against one launch per document on the same request streams."""
    import torch

    import gpupolyaurnlda_b200 as g
    from gpupolyaurnlda_b200 import corpus
    from gpupolyaurnlda_b200.serve import Server

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    c = corpus.generate("mid", seed=1, device=f"cuda:{local}")
    s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=0)
    s.corpus_load(c.z.copy(), c.w, c.d_len)
    s.corpus_sweep(args.serve_train)
    srv_b = Server(50, seed=0, max_inflight=1 << 17)  # persistent: 32 request warps per SM
    srv_u = Server(50, mode="launch", slots=args.serve_slots, max_batch=1, seed=0)
    q_model = s.read_state(n=False, alias=False, A=False, S=False, nnz=False)["q"]
    s.close()
    del c
    rows, ll = serve_measure(srv_b, srv_u, q_model, args.rates, args.serve_seconds, args.serve_requests,
                             args.serve_unbatched, local)
    st_b = srv_b.stats()
    srv_b.close()
    srv_u.close()
    top = rows[-1]
    if rank == 0:
        line = {"metric": "served_docs_per_sec", "value": top["batched"]["docs_per_sec"], "unit": "docs/s",
                "n_gpus": 1, "steps": len(rows), "warmup": 0,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u64", "data": "synthetic",
                "config": {"workload": f"serving fold-in: K=1000 V=100000 model (mid corpus, {args.serve_train} "
                                       f"training iterations), {SERVE_WORKLOAD} at {list(args.rates)} docs/s",
                           "batched": "persistent kernel, 32 request warps per SM",
                           "unbatched": f"one launch per document, {args.serve_slots} streams"},
                "p50_ms": top["batched"]["p50_ms"], "p99_ms": top["batched"]["p99_ms"],
                "unbatched": top["unbatched"],
                "speedup_vs_unbatched": top["batched"]["docs_per_sec"] / top["unbatched"]["docs_per_sec"],
                "heldout_ll_per_token": ll, "rates": rows, "server_stats": st_b}
        print(json.dumps(line), flush=True)


def run_sharded(args):
    """One chain, documents sharded across the ranks by token-balanced ranges;
    after every iteration the ranks add their count tables (NCCL all-reduce),
    so the chain equals the single-GPU chain.  value = corpus tokens per
    second of the whole job (strong scaling)."""
    import datetime

    import torch
    import torch.distributed as dist

    import gpupolyaurnlda_b200 as g
    from gpupolyaurnlda_b200.shard import LibraryShard, ShardedChain, shard_ranges

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            **({} if "MASTER_ADDR" in os.environ else
                               {"init_method": "tcp://127.0.0.1:29533", "rank": 0, "world_size": 1}))
    c = make_corpus(args, f"cuda:{local}")
    sh = shard_ranges(c.d_len, world)[rank]
    s = g.Sampler(c.alpha, c.beta, c.K, c.counts, buffer_size=16, max_D=4, seed=0)
    chain = ShardedChain(LibraryShard(s, c.z, c.w, c.d_len, sh))
    chain.iterate(args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    dist.barrier()
    t0 = time.perf_counter()
    chain.iterate(args.steps)
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0, f"cuda:{local}")
    clk = clocks.stop()
    s.close()
    if rank == 0:
        line = {"metric": METRIC, "value": c.n_tokens * args.steps / el, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic",
                "config": workload_desc(c, args), "parallelism": f"document shards x{world} + count all-reduce",
                "timing": "wall clock around the timed iterations (each ends with a host synchronisation), max over "
                          "ranks", "clocks": clk}
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.shard:
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
