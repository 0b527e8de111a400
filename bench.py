#!/usr/bin/env python
"""Gibbs tokens/s per sweep of the EZLDA collapsed-Gibbs sweep on the K=1024 workload.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Workload (one "step" = one full sweep: word-topic + topic-total rebuild, per-word max
topics, per-chunk doc-topic rebuild and sampling): a seeded synthetic corpus from the LDA
generative process standing in for EZLDA's PubMed run (EZLDA/mainKernel.cu:56; the data
are not available): D=300,000 docs, V=100,000 words, lognormal(5.3,0.6) doc lengths
clipped to [20,2000] (~71.9M tokens), 256 generating topics, Zipf(1.05) word base measure,
K=1024, alpha=50/K, beta=0.01, top-2% words dense, 8 chunks.  The K timed sweeps are
sweeps 0..K-1 of training from the random initial topics (the warm-up sweeps run first and
the topics are then reset), so the number is the average over a training run, early
(dense doc rows, few early accepts) and late sweeps alike.

--impl reference times the CPU restatement of the reference's sweep on the host cores.
EZLDA has no CPU implementation of its sampler, so that arm runs the oracle port
(oracle/liblda_oracle.c) with all host threads.  Its step is one whole sweep (count
rebuild + sampling of every token) of a bounded sample of the workload: 1/50 of the
documents drawn from the same generative process by a numpy generator
(oracle/sample_corpus.py), so that arm never loads the product library.  The cpu_baseline
leg of the default run uses the same definition (same sample, same sweeps).

Reference legs of the default run (baselines, never on the measured path):
  cpu_baseline   the oracle port as above;
  ezlda_b200     EZLDA's own kernels (oracle/_ref/ref_harness, built from the reference's
                 sources) timed on this B200 with their own events, against this library on
                 the same corpus, when the harness binary is present;
  serving        the fold-in serving figures (one at a time, saturated batch, offered loads).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "gibbs_tokens_per_s_per_iter"
UNIT = "tokens/s"
WORKLOADS = {
    "c1": ("lognormal K=1024 corpus: D=300000 V=100000 len~lognormal(5.3,0.6) in [20,2000] "
           "(~71.9M tokens), 256 generating topics, Zipf(1.05) phi base, alpha=50/K, beta=0.01, "
           "top-2% dense words, 8 chunks; sweeps 0..K-1 from random initial topics"),
    "c2": ("large-K corpus: D=1000000 V=1000000 len~Poisson(250) (~250M tokens), 1000 generating "
           "topics, Zipf(1.05) phi base (urn form), K=10000, alpha=0.1, beta=0.01, top-20000 dense "
           "words, 8 chunks; sweeps 0..K-1 from random initial topics"),
}
ALPHA = {"c2": 0.1, "c2s": 0.1}  # other presets: 50/K


def workload(preset: str) -> str:
    return WORKLOADS.get(preset, f"corpus preset {preset}")


HBM_FALLBACK_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-ezlda", action="store_true", help="skip the EZLDA-on-this-GPU reference leg")
    p.add_argument("--no-serving", action="store_true", help="skip the fold-in serving figures")
    p.add_argument("--preset", default="c1")
    p.add_argument("--chunks", type=int, default=0, help="override the preset's chunk count")
    p.add_argument("--sharded", action="store_true",
                   help="use the document-sharded path even on one GPU (it is the default for N>1)")
    p.add_argument("--stream", action="store_true",
                   help="stream the chunks through 4 CUDA streams (EZLDA's chunk streaming) instead of "
                        "keeping the corpus resident")
    p.add_argument("--budget-gb", type=float, default=0.0, help="device budget of the trainer (0: none)")
    p.add_argument("--batch", action="store_true",
                   help="batched multi-model benchmark: 512 small corpora in one graph-captured batch "
                        "against the same models trained one after another")
    p.add_argument("--batch-models", type=int, default=512)
    p.add_argument("--batch-sweeps", type=int, default=100)
    p.add_argument("--serve", action="store_true",
                   help="fold-in serving benchmark instead of the training sweep")
    p.add_argument("--serve-sweeps", type=int, default=30)
    p.add_argument("--serve-rates", default="2000,10000,50000", help="offered loads in docs/s")
    p.add_argument("--serve-seconds", type=float, default=1.5, help="arrival window per offered load")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"


def ncu_traffic(preset: str, tokens_per_launch: float):
    """Per-launch DRAM bytes (read + write) of the sampler: the bytes per token of a small
    ncu capture of the same kernel on the one-fifth K=1024 corpus
    (profiles/k_sample_c1s_traffic.json, a few launches), scaled by this run's tokens per
    launch.  The sampler's DRAM traffic is per-token data (token docs, metadata, topics)
    plus word columns; doc rows come from L2, so it grows with the tokens."""
    if preset not in ("c1", "c1s"):
        return None
    path = os.path.join(ROOT, "profiles", "k_sample_c1s_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        return {"dram_bytes_per_launch": float(t["dram_bytes_per_token"]) * tokens_per_launch,
                "source": f"profiles/k_sample_c1s_traffic.json ({t['dram_bytes_per_token']:.1f} B/token) "
                          f"x {tokens_per_launch:.0f} tokens per launch"}
    except (OSError, ValueError, KeyError):
        return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def physical_gpu(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local < len(ids) and ids[local].strip().isdigit():
            return int(ids[local])
    return local


def make_corpus(preset: str, rank: int, chunks: int = 0):
    import lda_sc20_b200 as L
    base = L.corpus_config(preset)
    over = {"corpus_seed": base.corpus_seed + rank}
    if chunks > 0:
        over["num_chunks"] = chunks
    return L.Corpus.generate(L.corpus_config(preset, **over))


def sampler_algorithmic_bytes(cnt, K: int, dense_words_per_sweep: int, sweeps: int, launches: int) -> float:
    """Algorithmic bytes of the sampler over the timed region: per token 16 B (doc id, old
    topic, new topic, doc length), 4 B per doc-row entry of every token whose S is evaluated,
    4*K per dense word column and 4 B per sparse word-row entry (per chunk launch), 4*K for
    n_k per launch."""
    return (16.0 * cnt.tokens + 4.0 * cnt.sum_nnz_full + 4.0 * K * dense_words_per_sweep * sweeps
            + 4.0 * cnt.sum_word_nnz + 4.0 * K * launches)


def run_sharded(args, world, rank, local):
    """N GPUs, one process each: the corpus is split by chunks (documents) for sampling and
    by word ranges for the word side, and the ranks exchange both every sweep
    (lda_sc20_b200.sharded).  Total work is fixed, so this is strong scaling."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    from lda_sc20_b200.sharded import ShardedTrainer

    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29533")
    os.environ.setdefault("RANK", str(rank))
    os.environ.setdefault("WORLD_SIZE", str(world))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    corpus = make_corpus(args.preset, 0, args.chunks)
    info = corpus.info
    K, N = info.K_hint, info.num_tokens
    st = ShardedTrainer(corpus, K=K, rank=rank, world=world, device=local, seed=42, alpha=ALPHA.get(args.preset))
    stream = torch.cuda.current_stream()
    z0 = corpus.topics()
    seg = corpus.seg_cnt()

    def reduce_max(x: float) -> float:
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = ClockSampler(physical_gpu(local))
    clocks.start()
    st.iterate(args.warmup)
    st.tr.set_topics(z0)
    st.tr.iteration = 0
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st.iterate(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    ms = reduce_max(e0.elapsed_time(e1))
    z_after = st.topics()
    h = torch.tensor([int(z_after[::101].astype(np.int64).sum())], dtype=torch.int64, device="cuda")
    hs = [torch.zeros_like(h) for _ in range(world)]
    dist.all_gather(hs, h)
    agree = all(int(x.item()) == int(h.item()) for x in hs)
    # the same sweeps again with per-stage CUDA events (stages one at a time on the
    # trainer's stream), for the stage split and the sampler's roofline
    st.tr.set_topics(z0)
    st.tr.iteration = 0
    st.tr.reset_stats()
    st.tr.set_timing(True)
    st.iterate(args.steps)
    torch.cuda.synchronize()
    tm = st.tr.timing()
    cnt = st.tr.counters()
    st.tr.set_timing(False)
    ll_mean = st.iterate(1, ll=True)
    # end to end: each rank uploads its chunks' topics, exchanges, sweeps, downloads its chunks
    e2e = None
    if not args.no_e2e:
        a, b = st.own_slice
        hin = torch.from_numpy(z0.view(np.int16)[a:b].copy()).pin_memory()
        hout = torch.empty_like(hin).pin_memory()
        st.tr.set_topics(z0)
        st.tr.iteration = 0
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st.z[a:b].copy_(hin, non_blocking=True)
            st.ex.exchange()
            st.sweep()
            hout.copy_(st.z[a:b])
            hin, hout = hout, hin
        torch.cuda.synchronize()
        e2e_s = reduce_max(time.perf_counter() - t0)
        e2e = {"value": N * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * (b - a),
               "d2h_bytes_per_step": 2 * (b - a), "ms_per_step": 1e3 * e2e_s / args.steps,
               "note": "per rank: its chunks' topics in and out, plus the in-place NCCL topic exchange"}
    launches = tm.launches_sample
    lo, hi = st.ranges[rank]
    dense_words = int((seg[lo:hi, :info.num_dense] > 0).sum())
    alg = sampler_algorithmic_bytes(cnt, K, dense_words, args.steps, launches)
    ms_launch = tm.ms_sample / max(launches, 1)
    achieved = alg / max(launches, 1) / (ms_launch / 1e3) / 1e9 if launches else None
    peaks, src = measured_peaks()
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
    if rank == 0:
        line = {
            "metric": METRIC, "value": N * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.preset, args.chunks), "tokens_per_step": N, "dense_words": info.num_dense,
            "run": {"parallelism": f"doc-sharded x{world}: chunks {st.ranges}, word ranges {st.word_ranges}; "
                                       "per sweep an n_k all-reduce, a word-side all-gather "
                                       f"({st.wx.bytes_per_rank} B per rank) and a topic all-gather"},
            "loglik_per_token": ll_mean, "ranks_agree": agree, "e2e": e2e,
            "gpu_launches": tm.launches_wt + tm.launches_stats + tm.launches_dt + tm.launches_sample + tm.launches_ll,
            "roofline": {"bound": "hbm", "kernel": "k_sample", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "peak_source": f"{src} hbm_gbs", "ms_per_launch": ms_launch, "rank": 0},
            "stages_ms_per_sweep": {"wt": tm.ms_wt / args.steps, "stats": tm.ms_stats / args.steps,
                                    "dt": tm.ms_dt / args.steps, "sample": tm.ms_sample / args.steps},
            "clocks": clk, "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    st.close()
    dist.barrier()
    dist.destroy_process_group()


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import lda_sc20_b200 as L

    if world > 1 or args.sharded:
        return run_sharded(args, world, rank, local)
    torch.cuda.set_device(local)
    corpus = make_corpus(args.preset, rank, args.chunks)
    info = corpus.info
    K = info.K_hint
    N = info.num_tokens
    tr = L.Trainer(corpus, K=K, seed=42, device=local, alpha=ALPHA.get(args.preset),
                   device_budget=int(args.budget_gb * 2**30), stream_mode=2 if args.stream else 0,
                   num_streams=4 if args.stream else 0)
    streaming, n_streams, _ = tr.stream_info()
    stream = torch.cuda.current_stream()
    tr.set_stream(stream.cuda_stream)
    z0 = corpus.topics()
    seg = corpus.seg_cnt()
    dense_words_per_sweep = int((seg[:, :info.num_dense] > 0).sum())

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def reduce_max(x: float) -> float:
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = ClockSampler(physical_gpu(local))
    clocks.start()
    tr.iterate(args.warmup)                      # untimed warm-up sweeps
    tr.set_topics(z0)                            # time sweeps 0..K-1 of a fresh run
    tr.iteration = 0
    tr.reset_stats()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tr.iterate(args.steps, ll=False)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    ms = reduce_max(ms_local)
    # the same sweeps again with per-stage CUDA events (stages run one at a time on the
    # trainer's stream then), for the stage split and the sampler's roofline
    tr.set_topics(z0)
    tr.iteration = 0
    tr.reset_stats()
    tr.set_timing(True)
    tr.iterate(args.steps, ll=False)
    torch.cuda.synchronize()
    tm = tr.timing()
    cnt = tr.counters()
    tr.set_timing(False)
    ms_staged = tm.ms_wt + tm.ms_stats + tm.ms_dt + tm.ms_sample
    device_bytes = tr.device_bytes
    streamed_gib = tr.stream_info()[2] / 2**30
    # log-likelihood of the state after the K timed sweeps (one extra evaluation sweep)
    z_after = tr.topics()
    ll_mean = tr.iterate(1, ll=True)
    # sweep time with the FP64 LL evaluated every sweep (LL mode evaluates S for all tokens),
    # beside plain sweeps over the same first sweeps (early sweeps cost more than the average)
    n_ll = max(1, min(args.steps, 10))
    ll_ms = {}
    for mode in (False, True):
        tr.set_topics(z0)
        tr.iteration = 0
        torch.cuda.synchronize()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        tr.iterate(n_ll, ll=mode)
        e3.record(stream)
        torch.cuda.synchronize()
        ll_ms[mode] = e2.elapsed_time(e3) / n_ll
    ms_ll_sweep = ll_ms[True]

    # per-sweep device time over a fresh run of the same sweeps (diagnostic, not the metric)
    tr.set_topics(z0)
    tr.iteration = 0
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        check_iter(tr, 1)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    per_sweep = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    marks = sorted({i for i in (0, 1, 2, 5, 10, 20, 50, 99, args.steps - 1) if i < args.steps})
    trace = {str(i): round(per_sweep[i], 3) for i in marks}

    sweeps = args.steps
    value = world * N * sweeps / (ms / 1e3)
    launches_sample = tm.launches_sample
    alg_bytes = sampler_algorithmic_bytes(cnt, K, dense_words_per_sweep, sweeps, launches_sample)
    ms_per_launch = tm.ms_sample / max(launches_sample, 1)
    achieved = alg_bytes / launches_sample / (ms_per_launch / 1e3) / 1e9 if launches_sample else None
    if streaming and K <= 2048:
        achieved = None  # the timed stage spans the chunk copies, doc-row rebuilds and sampling
    peaks, peak_src = measured_peaks()
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
    traffic = ncu_traffic(args.preset, cnt.tokens / max(launches_sample, 1))

    # end to end through the C ABI with pinned host buffers: upload topics, sweep, download
    e2e = None
    if not args.no_e2e:
        zin = torch.from_numpy(z0.view(np.int16).copy()).pin_memory()
        zout = torch.empty_like(zin).pin_memory()
        tr.iteration = 0
        tr.iterate_host_async(zin.numpy().view(np.uint16), zout.numpy().view(np.uint16))  # warm-up call
        tr.wait()
        tr.iteration = 0
        zin.copy_(torch.from_numpy(z0.view(np.int16)))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a, b = zin, zout
        for _ in range(sweeps):
            # each sweep uploads its input and downloads its output chunk by chunk; a chunk
            # of the next input goes up as soon as the previous sweep has brought it down
            tr.iterate_host_async(a.numpy().view(np.uint16), b.numpy().view(np.uint16))
            a, b = b, a
        tr.wait()
        t1 = time.perf_counter()
        barrier()
        e2e_s = reduce_max(t1 - t0)
        assert np.array_equal(a.numpy().view(np.uint16), z_after), "host-buffer sweeps diverged from resident sweeps"
        e2e = {"value": world * N * sweeps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * N,
               "d2h_bytes_per_step": 2 * N, "ms_per_step": 1e3 * e2e_s / sweeps}

    # fold-in serving against this corpus' model after 100 sweeps (the serving workload's
    # frozen word-topic counts)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving and args.preset == "c1" and not streaming:
        from lda_sc20_b200.serving import Model
        tr.set_topics(z0)
        tr.iteration = 0
        tr.iterate(100)
        model = Model(tr)
        serving = serving_figures(model, corpus, args.serve_sweeps, args.serve_rates, args.serve_seconds)
        model.close()
    tm_launches = tm.launches_wt + tm.launches_stats + tm.launches_dt + tm.launches_sample + tm.launches_ll
    tr.close()

    # reference legs (baselines; rank 0 of a one-GPU run only)
    cpu = None
    ezlda = None
    if rank == 0 and world == 1:
        if not args.no_cpu_baseline:
            c = cpu_sweeps(args.preset, args.warmup, sweeps)
            cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if not args.no_ezlda and K == 1024:
            ezlda = ezlda_leg()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": sweeps,
            "warmup": args.warmup, "ms_per_step": ms / sweeps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.preset, args.chunks),
            "tokens_per_step": N, "dense_words": info.num_dense,
            "run": {"parallelism": "single GPU", "device_bytes": device_bytes,
                    "chunks_streamed": (f"{n_streams} streams, {streamed_gib:.1f} GiB copied host->device in total")
                    if streaming else "no (resident)"},
            "loglik_per_token": ll_mean,
            "ms_per_step_with_ll": ms_ll_sweep,
            "ll_sweeps": {"sweeps": f"0-{n_ll - 1}", "plain_ms": ll_ms[False], "with_ll_ms": ll_ms[True],
                          "ll_cost": ll_ms[True] / ll_ms[False] - 1.0},
            "e2e": e2e,
            "gpu_launches": tm_launches,
            "roofline": {"bound": "hbm", "kernel": "k_sample", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic.get("dram_bytes_per_launch") if traffic else None,
                         "traffic_source": traffic.get("source") if traffic else None,
                         "peak_source": f"{peak_src} hbm_gbs",
                         "algorithmic_bytes_per_launch": alg_bytes / max(launches_sample, 1),
                         "ms_per_launch": ms_per_launch},
            "stages_ms_per_sweep": {"wt": tm.ms_wt / sweeps, "stats": tm.ms_stats / sweeps,
                                    "dt": tm.ms_dt / sweeps, "sample": tm.ms_sample / sweeps,
                                    "sum_staged": ms_staged / sweeps,
                                    "note": (("streamed: chunks rebuilt and sampled one after another; a slot "
                                              "stream copies ahead each chunk that no slot holds") if K > 2048 else
                                             ("streamed: 'sample' spans copies, doc-row rebuilds and sampling "
                                              "of all chunks on their streams")) if streaming else
                                            ("stages timed one at a time in a second pass over the same sweeps; "
                                             + ("the timed run samples the chunks one after another, each chunk's "
                                                "sparse-word sampler beside its dense-word one" if K > 2048 else
                                                "the timed run overlaps one chunk group's doc-topic rebuild and "
                                                "sampling with the other's"))},
            "sweep_ms_trace": trace,
            "sweep_counters": {"early_accept_frac": cnt.early_accept / max(cnt.tokens, 1),
                               "mean_nnz_full": cnt.sum_nnz_full / max(cnt.full, 1),
                               "rows_per_evaluated_token": cnt.rows_evaluated / max(cnt.full, 1),
                               "branch_max": cnt.branch_max, "branch_s": cnt.branch_s, "branch_q": cnt.branch_q},
            "clocks": clk,
            "cpu_baseline": cpu,
            "ezlda_b200": ezlda,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def check_iter(tr, n):
    """n sweeps enqueued without waiting (the C ABI call returns after its own sync)."""
    tr.iterate(n)


CPU_SAMPLE_DOC_FRACTION = 50  # the CPU legs sweep 1/50 of the preset's documents


def cpu_sweeps(preset: str, warmup: int, steps: int) -> dict:
    """The CPU leg: the oracle port, all host threads, timing whole sweeps (count rebuild +
    sampling of every token) of a sample corpus of 1/50 of the preset's documents, drawn
    from the same generative process.  `warmup` untimed sweeps, then `steps` timed ones
    from the sample's random initial topics (the same sweep indices the GPU arm times).
    Loads only the oracle library."""
    import numpy as np
    import lda_sc20_b200 as L  # presets only (pure Python; the native library is not loaded)
    from oracle import Oracle
    from oracle.sample_corpus import draw_corpus
    cfg = L.corpus_config(preset)
    D = max(1, cfg.num_docs // CPU_SAMPLE_DOC_FRACTION)
    c = draw_corpus(cfg, D, seed=int(cfg.corpus_seed) + 7)
    K = c["K"]
    alpha = ALPHA.get(preset, 50.0 / K)
    nt = os.cpu_count() or 1
    o = Oracle(c["tok_word"], c["tok_doc"], c["V"], c["D"], K, alpha, 0.01, nthreads=nt)
    z = c["topics"].copy()
    for it in range(warmup):
        o.iterate(z, 42, it)
    times = []
    for it in range(warmup, warmup + steps):
        t0 = time.perf_counter()
        o.iterate(z, 42, it)
        times.append(time.perf_counter() - t0)
    sec = float(np.mean(times))
    N = c["N"]
    return {"value": N / sec, "unit": UNIT, "cores": nt, "kind": "port", "ms_per_step": 1e3 * sec,
            "tokens_per_step": N,
            "sample": (f"whole sweeps (rebuild + sampling of every token) of a {D}-document, {N}-token corpus "
                       f"drawn by oracle/sample_corpus.py from the preset's generative process (1/"
                       f"{CPU_SAMPLE_DOC_FRACTION} of its documents); sweeps {warmup}..{warmup + steps - 1} "
                       f"after {warmup} untimed ones; {nt} threads; per-sweep seconds min/median/max "
                       f"{min(times):.3f}/{float(np.median(times)):.3f}/{max(times):.3f}")}


def workload_config(preset: str, chunks: int = 0) -> dict:
    """The workload both arms name: the preset's generator parameters (pure Python, no
    native library)."""
    import lda_sc20_b200 as L
    g = L.corpus_config(preset)
    return {"workload": workload(preset), "docs": int(g.num_docs), "vocab": int(g.vocab), "K": int(g.K),
            "alpha": float(ALPHA.get(preset, 50.0 / g.K)), "beta": 0.01, "corpus_seed": int(g.corpus_seed),
            "chunks": int(chunks or g.num_chunks),
            "l2": "inputs_larger_than_l2 (one sweep passes over the resident corpus, >1 GB, against a 126 MB L2)"}


def run_reference(args, world, rank, local):
    """CPU restatement of the reference sweep (oracle port), all host threads, rank 0 only."""
    if rank != 0:
        return
    cpu = cpu_sweeps(args.preset, args.warmup, args.steps)
    line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.preset, args.chunks), "impl": "reference",
            "tokens_per_step": cpu["tokens_per_step"],
            "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serving_figures(model, corpus, sweeps: int, rates_arg: str, seconds: float, n_batch: int = 60000) -> dict:
    """Fold-in serving against a frozen model: one request at a time (max_active=1, closed
    loop), a saturated batch (all requests queued at once), 32 batched requests again alone
    (same request ids, so the same randoms), and real-time replays of seeded Poisson
    arrivals at the offered loads with p50/p99 latency from scheduled arrival to theta on
    the host.  Requests are new documents from the corpus' generative process, lengths
    lognormal(median 150, sigma 1.0) in [5, 4000]; theta comes back as FP32[K]."""
    import numpy as np
    from lda_sc20_b200.serving import Server

    seed = 7
    rng = np.random.default_rng(11)
    req_seed = [1000]

    def requests(n):
        req_seed[0] += 1
        off, words = corpus.generate_requests(n, req_seed[0])
        return off, words, [words[off[i]:off[i + 1]] for i in range(n)]

    single = Server(model, sweeps=sweeps, max_active=1, max_tokens=1 << 16, seed=seed)
    _, _, docs1 = requests(300)
    single.run(docs1[:20])
    t0 = time.perf_counter()
    single.run(docs1)
    single_dps = len(docs1) / (time.perf_counter() - t0)
    single.close()
    batch = Server(model, sweeps=sweeps, max_active=16384, max_tokens=1 << 24, seed=seed)
    _, _, docsb = requests(n_batch)
    batch.run(docsb[:4000])
    s0, l0 = batch.stats()
    t0 = time.perf_counter()
    th_batch = batch.run(docsb)
    batch_s = time.perf_counter() - t0
    s1, l1 = batch.stats()
    batch_dps = len(docsb) / batch_s
    tokens_b = int(sum(len(d) for d in docsb))
    batch.close()
    alone = Server(model, sweeps=sweeps, max_active=1, max_tokens=1 << 16, seed=seed)
    ident = 0
    for i in range(32):
        alone.submit(i, docsb[i])
        while (r := alone.poll()) is None:
            alone.step()
        ident += int(np.array_equal(r[1].view(np.uint32), th_batch[i].view(np.uint32)))
    alone.close()
    rates = []
    for rate in [float(x) for x in rates_arg.split(",") if x]:
        n = max(1, int(rate * seconds))
        off, words, _ = requests(n)
        arrival = np.cumsum(rng.exponential(1.0 / rate, size=n))
        arrival -= arrival[0]
        srv = Server(model, sweeps=sweeps, max_active=16384, max_tokens=1 << 24, seed=seed)
        lat, _, wall = srv.replay(off, words, arrival)
        srv.close()
        rates.append({"offered_docs_per_s": rate, "requests": n, "achieved_docs_per_s": n / wall,
                      "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                      "max_ms": float(lat.max() * 1e3)})
    return {"docs_per_s": batch_dps, "one_at_a_time_docs_per_s": single_dps,
            "batch_vs_one_at_a_time": batch_dps / single_dps, "batch_token_sweeps_per_s": tokens_b * sweeps / batch_s,
            "batch_steps": s1 - s0, "gpu_launches": l1 - l0, "alone_equals_batched": f"{ident}/32",
            "rates": rates, "sweeps": sweeps}


def run_serving(args, local):
    """Fold-in serving against the word side of the K=1024 corpus trained for 100 sweeps
    (serving_figures)."""
    import torch
    import lda_sc20_b200 as L
    from lda_sc20_b200.serving import Model

    torch.cuda.set_device(local)
    corpus = make_corpus("c1", 0)
    info = corpus.info
    K = info.K_hint
    tr = L.Trainer(corpus, K=K, seed=42, device=local)
    tr.iterate(100)
    model = Model(tr)
    tr.close()
    clocks = ClockSampler(physical_gpu(local))
    clocks.start()
    f = serving_figures(model, corpus, args.serve_sweeps, args.serve_rates, args.serve_seconds)
    ck = clocks.stop()
    model.close()
    line = {"metric": "foldin_docs_per_s", "value": f["docs_per_s"], "unit": "docs/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"fold-in against the K={K} V={info.vocab} lognormal corpus trained 100 sweeps; "
                                   f"new documents from its generative process, lengths lognormal(median 150, "
                                   f"sigma 1.0) in [5,4000]; {f['sweeps']} sweeps per request; theta FP32[K]",
                       "sweeps": f["sweeps"], "K": K, "V": int(info.vocab)},
            **{k: v for k, v in f.items() if k not in ("docs_per_s", "sweeps")}, "clocks": ck}
    print(json.dumps(line), flush=True)


def ezlda_leg(sweeps: int = 30) -> dict:
    """EZLDA's own kernels timed on this B200 (oracle/_ref/ref_harness, built from the
    reference's sources; a baseline leg, never on the measured path) against this library
    on the same corpus: the largest shape EZLDA's sparse path takes (K=1024, no dense
    words, 8 chunks, ~14.5M tokens; its dense-word kernel, which claims segments with an
    unbounded cross-block spin lock, is never launched)."""
    import shutil
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"unavailable": "oracle/_ref/ref_harness is not built (no reference checkout where the build ran)"}
    from oracle.ref import run_ref
    tmp = tempfile.mkdtemp(prefix="ezlda_bench_")
    try:
        r = run_ref.ezlda_timing(tmp, sweeps)
    except Exception as e:  # a failed baseline leaves the measured numbers standing
        return {"unavailable": f"reference harness run failed: {e!r}"[:400]}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    p = run_ref.REF_TIME
    return {"corpus": (f"c1 process with D={p['num_docs']} V={p['vocab']} phi~Dir({p['phi_conc']}), K={run_ref.K}, "
                       f"no dense words, {p['num_chunks']} chunks, seed {p['corpus_seed']}"),
            "tokens": r["tokens"], "sweeps": r["sweeps"],
            "ref_ms_per_sweep": r["ref_ms_per_sweep"], "ref_ms_first_last": r["ref_ms_first_last"],
            "ours_ms": r["ours_ms_per_sweep"], "ours_e2e_ms": r["ours_e2e_ms_per_sweep"],
            "ratio": r["speedup_resident"], "e2e_ratio": r["speedup_e2e"], "ll_after": r["ll_after"],
            "host_sweeps_equal_resident": r["host_sweeps_equal_resident"],
            "timing": ("EZLDA: its own iterStart/iterStop CUDA events per sweep over its two-stream schedule "
                       "with every chunk copied host<->device (EZLDA/mainKernel.cu:344-347,376); ours: CUDA events "
                       "around resident sweeps, and wall clock around host-buffer sweeps"),
            "harness_wall_s": r["harness_wall_s"]}


def run_batch(args, local):
    """Batched training: args.batch_models independent corpora (K from {16,...,256}, D in
    [100,5000], V in [1000,20000], Poisson(80) lengths, 16 generating topics), each for
    args.batch_sweeps sweeps.  Plain: every model on its own trainer, one after another.
    Batched: the same models in one batch, autotuned, all sweeps in one graph launch.
    Every model's final topics must agree between the two."""
    from concurrent.futures import ThreadPoolExecutor
    import numpy as np
    import torch
    import lda_sc20_b200 as L
    from lda_sc20_b200.batch import Batch, batch_corpus_configs, dense_words_for, tune_dense_rule

    torch.cuda.set_device(local)
    cfgs = batch_corpus_configs(args.batch_models)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        corpora = list(ex.map(L.Corpus.generate, cfgs))
    Ks = [g.K for g in cfgs]
    N = [c.info.num_tokens for c in corpora]
    total = int(sum(N))
    sweeps = args.batch_sweeps
    clocks = ClockSampler(physical_gpu(local))
    clocks.start()
    plain = [L.Trainer(c, K=K, seed=11 + i, device=local) for i, (c, K) in enumerate(zip(corpora, Ks))]
    plain[0].iterate(1)                       # warm-up launch, then back to sweep 0
    plain[0].set_topics(corpora[0].topics())
    plain[0].iteration = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ll_plain = [t.iterate(sweeps, ll=True) for t in plain]
    plain_s = time.perf_counter() - t0
    # layout: the dense-word rule, picked on a sample of the models; then the batch's
    # launch tuning on the whole batch
    t0 = time.perf_counter()
    rule, rule_ms = tune_dense_rule(corpora, Ks, [11 + i for i in range(len(corpora))], device=local)
    batched = [L.Trainer(c, K=K, seed=11 + i, device=local, num_dense=dense_words_for(c, K, rule))
               for i, (c, K) in enumerate(zip(corpora, Ks))]
    b = Batch(batched)
    tuning, tuned_ms = b.autotune(sweeps_per_trial=2)
    tune_s = time.perf_counter() - t0
    l0, _ = b.stats()
    t0 = time.perf_counter()
    ll_b = b.iterate(sweeps, ll=True)
    batch_s = time.perf_counter() - t0
    l1, work = b.stats()
    clk = clocks.stop()
    same = sum(int(np.array_equal(p.topics(), q.topics())) for p, q in zip(plain, batched))
    ll_rel = max(abs(x - y) / abs(y) for x, y in zip(ll_b, ll_plain))
    line = {"metric": "batched_gibbs_tokens_per_s_per_iter", "value": total * sweeps / batch_s, "unit": "tokens/s",
            "n_gpus": 1, "steps": sweeps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(corpora)} independent corpora: K in {{16,32,64,128,256}}, D~U[100,5000], "
                                   f"V~U[1000,20000], len~Poisson(80), 16 generating topics, alpha=50/K, beta=0.01; "
                                   f"{sweeps} sweeps each", "models": len(corpora), "tokens": total},
            "plain_sequential_tokens_per_s": total * sweeps / plain_s,
            "batched_vs_plain": plain_s / batch_s,
            "seconds": {"plain_sequential": plain_s, "batched": batch_s, "autotune": tune_s},
            "autotune": {"warps": tuning[0], "schedule": ["largest_first", "model_major"][tuning[1]],
                         "tile_tokens": tuning[2], "ms_per_sweep": tuned_ms,
                         "dense_rule": {"None": "corpus split (count >= K)", "-1": "no dense words"}.get(
                             str(rule), f"count >= {rule}*K"),
                         "dense_rule_ms_per_sweep_on_sample": {str(k): round(v[0], 3) for k, v in rule_ms.items()}},
            "gpu_launches": l1 - l0, "work_items_per_sweep": work,
            "models_identical_to_plain": f"{same}/{len(corpora)}", "loglik_max_rel_diff": ll_rel,
            "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    if args.serve:
        return run_serving(args, local)
    if args.batch:
        return run_batch(args, local)
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
