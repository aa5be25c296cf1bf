"""Benchmark of the DF guiding hot path (guided queries/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload full|small]

A step is one gdf_infer over one bounce wavefront of synthetic query records
(default: 1920x1080 = 2,073,600 queries, 16-level 2^19 hash grids, 64x4
theta/phi MLPs, 64 bins each). `value` times the kernel with inputs resident
in HBM; `e2e` times the same call with host buffers, including the
host->device copy of the queries, guided mask and guiding data and the
device->host read of the guiding data. L2 is flushed (256 MiB write) between
timed steps, outside the timed events.

With --impl reference the CPU implementation of the same path runs on all
host cores, one whole bounce per step, with the same weights and query rows:
the reference's own interpolation and sampling code (train.h
thetaPostInference / phiPostInference, compiled for the host from the
reference tree) after a scalar fp32 forward of the same encodings and MLPs.

The side object `reference_gpu` times the reference's own GPU path --
tiny-cuda-nn v1.6 plus the reference DF kernels, rebuilt from the reference
tree for sm_100a (oracle/build_ref_gpu.py) -- on the same bounce and the same
training batch with the same weights, and the ratios of this library to it.

Multi-GPU: the path has no exchange step; each rank runs an independent
replica of the full workload (weak scaling), timed on the device, max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "guiding-df_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

FLOP_PER_QUERY = {  # 2 * sum(fan_in * fan_out), unpadded encoded widths, theta + phi
    "full": 2 * ((60 * 64 + 3 * 64 * 64 + 64 * 64) + (72 * 64 + 3 * 64 * 64 + 64 * 64)),
    "small": 2 * ((44 * 64 + 2 * 64 * 64 + 64 * 32) + (56 * 64 + 2 * 64 * 64 + 64 * 32)),
}
N_QUERIES = {"full": 1920 * 1080, "small": 65536}
TRAIN_BATCH = {"full": 262144, "small": 65536}
# training flops per record: forward + data gradient + weight gradient of
# both networks, 3x the forward (the backward's recomputation of the forward
# is an implementation cost, not counted)
TRAIN_FLOP_PER_RECORD = {k: 3 * v for k, v in FLOP_PER_QUERY.items()}
# MLP parameters of the theta + phi networks (tcnn pads input widths to 16);
# the rest of a network's parameters are its grid tables
MLP_PARAMS = {"full": (64 * 64 + 3 * 64 * 64 + 64 * 64) + (80 * 64 + 3 * 64 * 64 + 64 * 64),
              "small": (48 * 64 + 2 * 64 * 64 + 64 * 32) + (64 * 64 + 2 * 64 * 64 + 64 * 32)}
# grid-feature kernel, per query: the 3 position floats read, both networks'
# fp16 features written (2 x levels x features x 2 B); plus the fp16 tables once
FEATURE_BYTES_PER_QUERY = {"full": 12 + 2 * 16 * 2 * 2, "small": 12 + 2 * 8 * 2 * 2}
METRIC = "guided queries/s"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


def mlp_dims(cfg, net: int) -> list[tuple[int, int]]:
    """(rows, cols) of each MLP matrix of a DF network in tcnn order: first
    layer 64 x k0 (encoded width padded to 16), hidden 64 x 64, output rows
    padded to 16."""
    lf = cfg.grid_theta.n_levels * cfg.grid_theta.n_features_per_level
    k0 = (lf + 28 + (12 if net == 1 else 0) + 15) // 16 * 16
    h = cfg.mlp_theta.n_hidden_layers if net == 0 else cfg.mlp_phi.n_hidden_layers
    bins = cfg.n_bins_theta if net == 0 else cfg.n_bins_phi
    return [(64, k0)] + [(64, 64)] * (h - 1) + [((bins + 15) // 16 * 16, 64)]


def bench_weights(cfg, net: int, n_params: int, seed: int) -> np.ndarray:
    """The benchmark's network weights, from numpy only so that every arm
    (this library, the reference GPU path, the CPU baseline) runs the same
    ones: Xavier-uniform MLP matrices x 2.5 (peaked distributions, so the
    sampling does real work) and grid tables U(-0.5, 0.5)."""
    rng = np.random.default_rng(seed * 2 + net)
    parts = []
    for r, c in mlp_dims(cfg, net):
        a = 2.5 * np.sqrt(6.0 / (r + c))
        parts.append(rng.uniform(-a, a, r * c))
    n_mlp = sum(r * c for r, c in mlp_dims(cfg, net))
    parts.append(rng.uniform(-0.5, 0.5, n_params - n_mlp))
    return np.concatenate(parts).astype(np.float32)


def workload_config(workload: str):
    """The networks of a workload as plain values (what the CPU arm needs,
    without loading this library): hash grids with tcnn's default base
    resolution 16 and per-level scale 2, SH degree 4, OneBlob 4 bins,
    TriangleWave 12 frequencies, linear pdf interpolation."""
    from types import SimpleNamespace as NS
    full = workload == "full"
    grid = NS(type=0, n_levels=16 if full else 8, n_features_per_level=2, log2_hashmap_size=19 if full else 16,
              base_resolution=16, per_level_scale=2.0, interpolation=0)
    mlp = NS(n_neurons=64, n_hidden_layers=4 if full else 3)
    bins = 64 if full else 32
    return NS(n_bins_theta=bins, n_bins_phi=bins, pdf_interp=0, grid_theta=grid, grid_phi=grid, sh_degree=4,
              oneblob_bins=4, tw_frequencies=12, mlp_theta=mlp, mlp_phi=mlp)


def bench_config(workload: str, precision: int = 0):
    """The library's preset for the workload, checked against workload_config."""
    import pygdf
    cfg = pygdf.default_config(pygdf.PRESET_FULL if workload == "full" else pygdf.PRESET_SMALL)
    cfg.precision = precision
    ref = workload_config(workload)
    for k in ("n_bins_theta", "n_bins_phi", "pdf_interp", "sh_degree", "oneblob_bins", "tw_frequencies"):
        assert getattr(cfg, k) == getattr(ref, k), k
    for g in ("grid_theta", "grid_phi"):
        for k in vars(ref.grid_theta):
            assert abs(getattr(getattr(cfg, g), k) - getattr(ref.grid_theta, k)) < 1e-6, (g, k)
    for m in ("mlp_theta", "mlp_phi"):
        for k in vars(ref.mlp_theta):
            assert getattr(getattr(cfg, m), k) == getattr(ref.mlp_theta, k), (m, k)
    return cfg


def make_context(workload: str, seed: int, precision: int = 0):
    import pygdf
    cfg = bench_config(workload, precision)
    ctx = pygdf.Context(cfg)
    params = []
    for net in (0, 1):
        p = bench_weights(cfg, net, ctx.n_params(net), seed)
        ctx.set_params(net, p)
        params.append(p)
    return ctx, cfg, params


def cpu_inputs(n: int, seed: int):
    """Query rows, guiding data, guided mask and uniforms of a bounce."""
    from pygdf import workload as W
    q = W.queries(n, seed)
    wi, guided = W.wi_init(n, seed, guided_frac=0.7, one_sided_frac=0.1)
    u = W.uniforms(n, seed)
    return q, wi, guided, u


def cpu_reference(cfg, params, inputs, threads: int):
    """The CPU baseline on one batch of queries: the reference's
    thetaPostInference / phiPostInference compiled for the host
    (oracle/_ref/libgdf_refcpu_*.so) after a scalar fp32 forward of the same
    encodings and MLPs. Returns (queries/s, queries, seconds)."""
    import oracle as O
    d = O.df_cfg_from(cfg)
    p16 = [O.round_f16(p) for p in params]
    q, wi, guided, u = inputs
    t0 = time.perf_counter()
    O.refcpu_infer(d, p16[0], p16[1], q, wi, guided, u, threads)
    el = time.perf_counter() - t0
    return q.shape[0] / el, q.shape[0], el


def cpu_sample(cfg, params, seconds: float, threads: int, chunk: int = 131072):
    """A bounded sample (about `seconds` of CPU work) of the CPU baseline on
    the bounce's first `chunk` queries, repeated."""
    inputs = cpu_inputs(chunk, 42)
    cpu_reference(cfg, params, tuple(x[:1024] for x in inputs), threads)  # warm
    done, el = 0, 0.0
    while el < seconds:
        _, k, t = cpu_reference(cfg, params, inputs, threads)
        done += k
        el += t
    return done / el, done, el


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="full", choices=["full", "small"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU-baseline sample length; 0 skips it (profiling runs)")
    ap.add_argument("--skip-e2e", action="store_true", help="profiling runs: kernel timing only")
    ap.add_argument("--serve-reserve", type=int, default=0,
                    help="serving stage: SMs training leaves to inference (gdf_server_config.train_sm_reserve)")
    ap.add_argument("--queries", type=int, default=0,
                    help="profiling runs: a smaller bounce of this many queries (0: the workload's)")
    ap.add_argument("--stages", default="infer,train,refgpu,records,forms,grouped,serve",
                    help="comma list of infer, train, records (profiling runs select one)")
    args = ap.parse_args()
    stages = set(args.stages.split(","))

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    n = args.queries if args.queries > 0 else N_QUERIES[args.workload]
    workload_name = ("DF guided inference, 1920x1080 wavefront: hash grid 16 levels x 2 features, "
                     "2^19 entries/level, theta/phi MLP 64x4, 64 bins, linear interpolation"
                     if args.workload == "full" else
                     "DF guided inference, 65,536 queries: hash grid 8x2, 2^16, MLP 64x3, 32 bins")
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # The reference's own CPU implementation of the path: its epilogue
        # (train.h) compiled for the host after a scalar fp32 forward of the
        # same networks, on every host thread; each step is one whole bounce
        # with this arm's weights and inputs.
        if rank != 0:
            return
        import oracle as O
        cfg = workload_config(args.workload)
        d = O.df_cfg_from(cfg)
        params = [bench_weights(cfg, net, O.df_n_params(d, net), 1234) for net in (0, 1)]
        inputs = cpu_inputs(n, 42)
        for _ in range(args.warmup):
            cpu_reference(cfg, params, inputs, threads)
        vals = [cpu_reference(cfg, params, inputs, threads) for _ in range(args.steps)]
        ms = statistics.mean(x[2] for x in vals) * 1e3
        v = n / (ms * 1e-3)
        sample = (f"the whole {n}-query bounce per step, {threads} threads: reference epilogue (train.h "
                  f"thetaPostInference / phiPostInference compiled for the host) after a scalar fp32 forward of "
                  f"the same encodings and MLPs, same weights and inputs as the GPU arm")
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": workload_name, "queries": n},
                "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from pygdf import workload as W
    ctx, cfg, params = make_context(args.workload, seed=1234 + rank)
    dev = torch.device("cuda", local_rank)
    q_h = W.queries(n, 42 + rank)
    wi_h, guided_h = W.wi_init(n, 42 + rank, guided_frac=0.7, one_sided_frac=0.1)
    q = torch.from_numpy(q_h).to(dev)
    wi0 = torch.from_numpy(wi_h).to(dev)
    guided = torch.from_numpy(guided_h).to(dev)
    wi = wi0.clone()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step(offset, stages=None):
        ctx.infer_ex(wi, n=n, queries=q, guided=guided, seed=7, offset=offset, stream=stream,
                     stage_events=stages)

    for i in range(args.warmup):
        wi.copy_(wi0)
        step(i)
    torch.cuda.synchronize()
    ctx.sync(stream)

    # ---- device-resident timing (kernel only, L2 flushed between steps)
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    times, stage_ms = [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        wi.copy_(wi0)
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # the call re-records these after its grid-feature and fused launches
        mid = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for m_ in mid:
            m_.record(stream)
        s.record(stream)
        step(1000 + i, mid)
        e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
        stage_ms.append((s.elapsed_time(mid[0]), mid[0].elapsed_time(mid[1])))
    torch.cuda.synchronize()
    ctx.sync(stream)
    if dist:
        dist.barrier()

    # ---- end to end through the C ABI with host buffers
    q_pin = torch.from_numpy(q_h).pin_memory()
    wi_pin = torch.from_numpy(wi_h).pin_memory()
    g_pin = torch.from_numpy(guided_h).pin_memory()
    out_pin = torch.empty_like(wi_pin).pin_memory()
    e2e_times = []
    for i in range(0 if args.skip_e2e else args.warmup + args.steps):
        # gdf_infer_host: host inputs in, guiding data out, copies pipelined
        # with the kernels inside the call
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        ctx.infer_host(q_pin, wi_pin, out_pin, guided=g_pin, seed=7, offset=5000 + i, n=n, stream=stream)
        e.record(stream)
        e.synchronize()
        if i >= args.warmup:
            e2e_times.append(s.elapsed_time(e))
    # the box's pinned-copy bandwidth, timed on the step's own pinned buffers:
    # the floor of the end-to-end step (its copies, one direction at a time)
    pcie = None
    if e2e_times:
        srcs = (q_pin, wi_pin, g_pin)
        dsts = tuple(torch.empty_like(x, device=dev) for x in srcs)
        pcie = {}
        for name in ("h2d", "d2h"):
            ts = []
            for _ in range(6):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    s.record(stream)
                    if name == "h2d":
                        for d_, h_ in zip(dsts, srcs):
                            d_.copy_(h_, non_blocking=True)
                    else:
                        out_pin.copy_(dsts[1], non_blocking=True)
                    e.record(stream)
                e.synchronize()
                ts.append(s.elapsed_time(e))
            nbytes = sum(x.nbytes for x in srcs) if name == "h2d" else out_pin.nbytes
            pcie[name + "_gbs"] = nbytes / (min(ts[2:]) * 1e-3) / 1e9
        del dsts
    # ---- training step (gdf_train_step on one batch of synthetic records)
    nb = TRAIN_BATCH[args.workload]
    train_times, rec_times, last, n_rec, rec_bytes = [], [], None, 0, 0
    if "train" in stages:
        train_times, last = time_train(ctx, cfg, W, nb, rank, dev, stream, flush, args)
    refgpu = None
    if "refgpu" in stages:
        refgpu = time_reference_gpu(ctx, cfg, params, q, wi0, guided, nb, rank, dev, stream, flush, args,
                                    statistics.mean(times),
                                    statistics.mean(train_times) if train_times else None)
    if "records" in stages:
        rec_times, n_rec, rec_bytes = time_records(ctx, W, n, rank, dev, stream, flush, args)
    form_times = {}
    if "forms" in stages:
        # the same bounce with the bf16 and FP8 inference forms (and the bf16
        # form's training step)
        import pygdf
        for name, prec in (("bf16", pygdf.PREC_BF16), ("fp8", pygdf.PREC_FP8)):
            cb, cfg_b, _ = make_context(args.workload, seed=1234 + rank, precision=prec)
            for i in range(args.warmup):
                wi.copy_(wi0)
                cb.infer(q, wi, guided=guided, seed=7, offset=i, n=n, stream=stream)
            ts = []
            for i in range(args.steps):
                wi.copy_(wi0)
                flush.zero_()
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                cb.infer(q, wi, guided=guided, seed=7, offset=1000 + i, n=n, stream=stream)
                e.record(stream)
                e.synchronize()
                ts.append(s.elapsed_time(e))
            form_times[name] = ts
            if name == "bf16" and "train" in stages:
                # the bf16 form trains in bf16 as well
                tt, _ = time_train(cb, cfg_b, W, nb, rank, dev, stream, flush, args)
                form_times["bf16_train"] = tt
            cb.sync(stream)
            cb.close()
    grouped = None
    if "grouped" in stages and args.workload == "full":
        grouped = time_grouped(W, rank, dev, stream, flush, args)
    serving = None
    if "serve" in stages and args.workload == "full":
        serving = time_serving(W, rank, dev, args)
    clk = clocks.stop()
    ctx.sync(stream)
    kern = {"stage_ms": stage_ms,
            "grid_bytes": 2 * (ctx.n_params(0) + ctx.n_params(1) - MLP_PARAMS[args.workload])}
    _report(args, rank, world, dist, dev, n, cfg, params, times, e2e_times, train_times, rec_times,
            last, n_rec, rec_bytes, clk, nb, workload_name, threads, q_h, wi_h, guided_h, form_times,
            grouped, serving, pcie, refgpu, kern)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def time_grouped(W, rank, dev, stream, flush, args):
    """8 render jobs with their own networks (4 with 64 bins, 4 with 32), 6
    bounces with wavefronts round(2,073,600 * 0.7^b): one grouped launch per
    bounce for all jobs, against the same work as separate gdf_infer calls."""
    import torch
    import pygdf
    n0, jobs_n, bounces = 2073600, 8, 6
    sizes = [int(round(n0 * 0.7 ** b)) for b in range(bounces)]
    ctxs, qs, wis, wi0s, gs = [], [], [], [], []
    for k in range(jobs_n):
        cfg = pygdf.default_config(pygdf.PRESET_FULL)
        cfg.n_bins_theta = cfg.n_bins_phi = 64 if k < 4 else 32
        ctxs.append(pygdf.Context(cfg))
        qs.append(torch.from_numpy(W.queries(n0, 500 + 7 * rank + k)).to(dev))
        wi_h, g_h = W.wi_init(n0, 500 + k, guided_frac=0.7, one_sided_frac=0.1)
        wi0s.append(torch.from_numpy(wi_h).to(dev))
        gs.append(torch.from_numpy(g_h).to(dev))
        wis.append([torch.empty((nb, 4), dtype=torch.float32, device=dev) for nb in sizes])
    group = pygdf.Group(max_jobs=jobs_n)

    def reset():
        for k in range(jobs_n):
            for b, nb in enumerate(sizes):
                wis[k][b].copy_(wi0s[k][:nb])

    def frame(grouped, f):
        for b, nb in enumerate(sizes):
            if grouped:
                group.infer([{"ctx": ctxs[k], "queries": qs[k], "wi": wis[k][b], "guided": gs[k], "n": nb,
                              "seed": 9, "offset": 100 * f + b} for k in range(jobs_n)], stream=stream)
            else:
                for k in range(jobs_n):
                    ctxs[k].infer(qs[k], wis[k][b], guided=gs[k], seed=9, offset=100 * f + b, n=nb,
                                  stream=stream)

    out = {}
    for name, grouped in (("grouped", True), ("separate", False)):
        for f in range(max(args.warmup, 1)):
            reset()
            frame(grouped, f)
        times = []
        for f in range(args.steps):
            reset()
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            frame(grouped, 1000 + f)
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
        out[name] = statistics.mean(times)
    group.sync(stream)
    wgs, fb, tune_ms = group.tuning()
    small = time_grouped_small(W, rank, dev, stream, flush, args)
    total = jobs_n * sum(sizes)
    res = {"metric": "guided queries/s, 8 jobs x 6 bounces in grouped launches",
           "value": total / (out["grouped"] * 1e-3), "unit": "queries/s", "ms_per_frame": out["grouped"],
           "separate_calls_ms_per_frame": out["separate"], "speedup_vs_separate": out["separate"] / out["grouped"],
           "queries_per_frame": total, "wavefronts": sizes, "bins": "4 jobs x 64, 4 jobs x 32",
           "launches_per_frame": 2 * bounces, "tuned": {"warpgroups": wgs, "feature_block": fb},
           "small_jobs": small}
    group.close()
    for c in ctxs:
        c.close()
    return res


def time_reference_gpu(ctx, cfg, params, q, wi0, guided, nb, rank, dev, stream, flush, args, ms_ours,
                       ms_ours_train):
    """The reference's own GPU path on this box: tiny-cuda-nn v1.6 and the
    reference DF kernels rebuilt for sm_100a (oracle/_ref/libgdf_tcnnref_*),
    with this arm's weights. Inference: the same bounce, query rows and
    guided mask, with explicit uniforms (the reference draws from a per-pixel
    sampler in memory; this library is also timed on the same explicit
    uniforms). Training: one batch of the same size as the `train` object."""
    import torch
    import oracle as O
    import tcnnref as T
    from pygdf import workload as W
    if not T.available(cfg.n_bins_theta, cfg.n_bins_phi):
        return {"unavailable": "reference GPU harness not built (oracle/build_ref_gpu.py)"}
    R = T.DfRef(cfg, scrub=False)
    for net in (0, 1):
        R.set_params(net, params[net])
    n = q.shape[0]
    u = torch.from_numpy(O.philox_uniforms(7, 0, n)).to(dev)
    wi = wi0.clone()
    sp = stream.cuda_stream

    def timed(fn, reps, warm):
        for _ in range(warm):
            wi.copy_(wi0)
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            wi.copy_(wi0)
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e))
        return statistics.mean(ts)

    ms_ref = timed(lambda: R.infer(wi, u, queries=q, guided=guided, stream=sp), args.steps, args.warmup)
    ms_same_u = timed(lambda: ctx.infer(q, wi, guided=guided, uniforms=u, n=n, stream=stream), args.steps,
                      args.warmup)
    ta, tb, tt = W.training_batch(nb, 77 + rank, cfg.n_bins_theta)
    da, db, dt = (torch.from_numpy(x).to(dev) for x in (ta, tb, tt))
    ms_ref_train = timed(lambda: R.train_step(da, db, dt, stream=sp), args.steps, args.warmup)
    R.close()
    return {"what": "tiny-cuda-nn v1.6 + reference DF kernels (train.h / train.cu), rebuilt from the reference "
                    "tree for sm_100a; LearnedDistribution::inferenceStep and one trainStep batch, same weights",
            "infer_ms": ms_ref, "infer_queries_s": n / (ms_ref * 1e-3),
            "ours_same_uniforms_ms": ms_same_u,
            "ratio_infer": ms_ref / ms_ours, "ratio_infer_same_uniforms": ms_ref / ms_same_u,
            "train_ms": ms_ref_train, "train_records_s": nb / (ms_ref_train * 1e-3),
            "ratio_train": ms_ref_train / ms_ours_train if ms_ours_train else None,
            "batch": nb, "queries": n}


def time_grouped_small(W, rank, dev, stream, flush, args):
    """Many small, uneven jobs -- the case grouping is for: 64 render jobs
    with their own networks (config-1 sizes, 32 or 64 bins) and wavefronts
    log-uniform in 2^10..2^16 queries, one grouped call against 64 separate
    gdf_infer calls."""
    import torch
    import pygdf
    n_jobs = 64
    rng = np.random.default_rng(700 + rank)
    sizes = [int(np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 16)))) for _ in range(n_jobs)]
    ctxs, qs, wis, wi0s, gs = [], [], [], [], []
    for k in range(n_jobs):
        cfg = pygdf.default_config(pygdf.PRESET_FULL)
        cfg.n_bins_theta = cfg.n_bins_phi = 64 if k % 2 == 0 else 32
        cfg.max_queries = 1 << 16
        ctxs.append(pygdf.Context(cfg))
        qs.append(torch.from_numpy(W.queries(sizes[k], 900 + 7 * rank + k)).to(dev))
        wi_h, g_h = W.wi_init(sizes[k], 900 + k, guided_frac=0.7, one_sided_frac=0.1)
        wi0s.append(torch.from_numpy(wi_h).to(dev))
        wis.append(torch.from_numpy(wi_h).to(dev))
        gs.append(torch.from_numpy(g_h).to(dev))
    group = pygdf.Group(max_jobs=n_jobs)

    def run(grouped, f):
        for k in range(n_jobs):
            wis[k].copy_(wi0s[k])
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        if grouped:
            group.infer([{"ctx": ctxs[k], "queries": qs[k], "wi": wis[k], "guided": gs[k], "n": sizes[k],
                          "seed": 9, "offset": f} for k in range(n_jobs)], stream=stream)
        else:
            for k in range(n_jobs):
                ctxs[k].infer(qs[k], wis[k], guided=gs[k], seed=9, offset=f, n=sizes[k], stream=stream)
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e)

    out = {}
    for name, grouped in (("grouped", True), ("separate", False)):
        for f in range(max(args.warmup, 1)):
            run(grouped, f)
        ts = []
        for f in range(args.steps):
            flush.zero_()
            ts.append(run(grouped, 1000 + f))
        out[name] = statistics.mean(ts)
    group.sync(stream)
    wgs, fb, _ = group.tuning()
    group.close()
    for c in ctxs:
        c.close()
    total = sum(sizes)
    return {"jobs": n_jobs, "queries": total, "sizes": "log-uniform 2^10..2^16 (seeded)",
            "ms_grouped": out["grouped"], "ms_separate": out["separate"],
            "speedup_vs_separate": out["separate"] / out["grouped"],
            "value": total / (out["grouped"] * 1e-3), "unit": "queries/s",
            "tuned": {"warpgroups": wgs, "feature_block": fb}}


SERVE_SLOTS, SERVE_TRAIN_SLOTS, SERVE_RUNS = 8, 2, 3


def time_serving(W, rank, dev, args):
    """64 resident instances (config-1 networks, 32 or 64 bins), requests of
    log-uniform size in [2^10, 2^21] queries, 1 training to 3 inference, under
    a 120 GB budget: a saturating burst gives the batched peak; Poisson
    arrivals at 80 % of it give the latency percentiles."""
    import time
    import torch
    import pygdf
    n_inst, n_max = 64, 1 << 21
    train_max = n_max
    insts = []
    for k in range(n_inst):
        cfg = pygdf.default_config(pygdf.PRESET_FULL)
        cfg.n_bins_theta = cfg.n_bins_phi = 64 if k % 2 == 0 else 32
        cfg.max_queries = n_max
        cfg.max_train_batch = train_max
        insts.append(pygdf.Context(cfg))
    budget = 120 * (1 << 30)
    srv = pygdf.Server(budget, slots=SERVE_SLOTS, max_batch=32, max_train_slots=SERVE_TRAIN_SLOTS,
                       train_sm_reserve=args.serve_reserve)
    for c in insts:
        srv.add_instance(c)
    q = torch.from_numpy(W.queries(n_max, 800 + rank)).to(dev)
    g = torch.from_numpy(W.wi_init(n_max, 800, guided_frac=0.7)[1]).to(dev)
    wi0 = torch.from_numpy(W.wi_init(n_max, 800, guided_frac=0.7)[0]).to(dev)
    # four output buffers per instance in turn: inference requests of one
    # instance may run together
    wis = [[wi0.clone() for _ in range(4)] for _ in range(n_inst)]
    tb = {}
    for bins in (32, 64):
        tb[bins] = tuple(torch.from_numpy(x).to(dev) for x in W.training_batch(train_max, 801, bins))
    rng = np.random.default_rng(900 + rank)

    def draw(m):
        out = []
        for _ in range(m):
            n = int(np.exp(rng.uniform(np.log(1 << 10), np.log(n_max))))
            out.append((int(rng.integers(n_inst)), n, rng.random() < 0.25))
        return out

    def submit(k, n, train, i):
        c = insts[k]
        if train:
            bins = c.cfg.n_bins_theta
            n = min(n, train_max)
            return srv.submit_train(c, tb[bins][0], tb[bins][1], tb[bins][2], n=n)
        return srv.submit_infer(c, q, wis[k][i % 4], guided=g, seed=k, offset=i, n=n)

    # warm-up: every graph shape and every instance's first requests
    for t in [submit(*r, i) for i, r in enumerate(draw(3 * n_inst))]:
        srv.wait(t)
    srv.stats(reset=True)
    # batched peak: bursts of requests submitted at once; how well one
    # burst batches varies (its order of sizes and instances), so the peak
    # is the median of three
    peaks, means = [], []
    for rep in range(3):
        burst = draw(400)
        for t in [submit(*r, 20000 * (rep + 1) + i) for i, r in enumerate(burst)]:
            srv.wait(t)
        pk = srv.stats(reset=True)
        peaks.append((pk.queries_per_s, pk.resident_bytes))
        means.append(float(np.mean([min(n, train_max) if tr else n for _, n, tr in burst])))
    peak_qps = float(np.median([p_[0] for p_ in peaks]))
    peak = type("Peak", (), {"queries_per_s": peak_qps, "resident_bytes": peaks[0][1]})
    mean_n = float(np.mean(means))
    rate = 0.8 * peak.queries_per_s / mean_n  # requests per second
    # isolated service time by kind, bin count and size (one request at a time)
    inf_sizes = [1 << e for e in range(10, 22)]
    trn_sizes = [1 << e for e in range(10, 22)]
    iso = {}
    for train, sizes in ((False, inf_sizes), (True, trn_sizes)):
        for k in (0, 1):  # even instances have 64 bins, odd ones 32
            iso[(train, k)] = [min(srv.wait(submit(k, n, train, 50000 + r))[1] for r in range(3)) for n in sizes]

    def iso_ms(k, n, train):
        sizes = trn_sizes if train else inf_sizes
        n = min(n, train_max) if train else n
        return float(np.exp(np.interp(np.log(n), np.log(sizes), np.log(iso[(train, k % 2)]))))

    def pct(x):
        return {"p50": float(np.percentile(x, 50)), "p99": float(np.percentile(x, 99))}

    runs = []
    # one Poisson run first, not reported: the slots' feature buffers and
    # launch graphs grow to this load's batch sizes
    for rep in range(-1, SERVE_RUNS):
        srv.stats(reset=True)
        reqs = draw(1000)
        tickets, t_sub = [], []
        t0 = time.perf_counter()
        next_t = t0
        for i, r in enumerate(reqs):
            next_t += rng.exponential(1.0 / rate)
            while time.perf_counter() < next_t:
                pass
            t_sub.append(time.perf_counter())
            tickets.append(submit(*r, 10000 * (rep + 2) + i))
        lat = np.array([srv.wait(t)[1] for t in tickets])
        st = srv.stats(reset=True)
        slow = lat / np.array([iso_ms(k, n, tr) for k, n, tr in reqs])
        is_tr = np.array([tr for _, _, tr in reqs])
        # requests that found an earlier request of their own instance still
        # in flight (same networks: they run in submission order)
        t_sub = np.array(t_sub)
        t_done = t_sub + lat * 1e-3
        queued = np.zeros(len(reqs), bool)
        last_done = {}
        for i, (k, _, _) in enumerate(reqs):
            queued[i] = last_done.get(k, -1.0) > t_sub[i]
            last_done[k] = max(last_done.get(k, -1.0), t_done[i])
        if rep < 0:
            continue
        runs.append({"p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms,
                     "p99_over_p50": st.p99_ms / st.p50_ms if st.p50_ms > 0 else None,
                     "slowdown": {**pct(slow), "p99_over_p50": float(np.percentile(slow, 99) / np.percentile(slow, 50))},
                     "inference_ms": pct(lat[~is_tr]), "training_ms": pct(lat[is_tr]),
                     "behind_own_instance": {"requests": int(queued.sum()),
                                             "slowdown": pct(slow[queued]) if queued.any() else None,
                                             "slowdown_of_the_rest": pct(slow[~queued])},
                     "throughput": st.queries_per_s, "frac_of_peak": st.queries_per_s / peak.queries_per_s,
                     "requests": st.requests})

    def med(f):
        return float(np.median([f(r) for r in runs]))

    def spread(f):
        v = [f(r) for r in runs]
        return [float(min(v)), float(max(v))]

    res = {"metric": "serving: 64 instances, Poisson arrivals, continuous batching",
           "runs": len(runs), "reported": "median over the runs; *_range = [min, max] over the runs",
           "p50_ms": med(lambda r: r["p50_ms"]), "p99_ms": med(lambda r: r["p99_ms"]),
           "p99_over_p50": med(lambda r: r["p99_over_p50"]),
           "p99_over_p50_range": spread(lambda r: r["p99_over_p50"]),
           "slowdown": {"p50": med(lambda r: r["slowdown"]["p50"]), "p99": med(lambda r: r["slowdown"]["p99"]),
                        "p99_range": spread(lambda r: r["slowdown"]["p99"]),
                        "definition": "latency / the same request's isolated latency (same kind, bins, size)"},
           "inference_ms": {"p50": med(lambda r: r["inference_ms"]["p50"]),
                            "p99": med(lambda r: r["inference_ms"]["p99"])},
           "training_ms": {"p50": med(lambda r: r["training_ms"]["p50"]),
                           "p99": med(lambda r: r["training_ms"]["p99"])},
           "throughput": med(lambda r: r["throughput"]), "unit": "queries/s",
           "batched_peak": peak.queries_per_s, "batched_peak_bursts": [p_[0] for p_ in peaks], "frac_of_peak": med(lambda r: r["frac_of_peak"]),
           "frac_of_peak_range": spread(lambda r: r["frac_of_peak"]),
           "offered_load": "80 % of the batched peak", "requests_per_run": 1000,
           "resident_gb": peak.resident_bytes / 2 ** 30, "budget_gb": budget / 2 ** 30,
           "sizes": "log-uniform 2^10..2^21 queries or training records",
           "mix": "1 training : 3 inference", "train_sm_reserve": args.serve_reserve,
           "per_run": runs}
    srv.close()
    for c in insts:
        c.close()
    return res


def time_train(ctx, cfg, W, nb, rank, dev, stream, flush, args):
    import torch
    ta, tb, tt = W.training_batch(nb, 77 + rank, cfg.n_bins_theta)
    da, db, dt = (torch.from_numpy(x).to(dev) for x in (ta, tb, tt))
    for _ in range(args.warmup):
        ctx.train_step(da, db, dt, stream=stream, stats=False)
    torch.cuda.synchronize()
    train_times = []
    for i in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        ctx.train_step(da, db, dt, stream=stream, stats=False)
        e.record(stream)
        e.synchronize()
        train_times.append(s.elapsed_time(e))
    last = ctx.train_step(da, db, dt, stream=stream, stats=True)
    return train_times, last


def time_records(ctx, W, n, rank, dev, stream, flush, args):
    """training-record producer (gdf_build_train_records) over one frame"""
    import torch
    import pygdf
    n_px = n
    fields, depth = W.path_state(n_px, 91 + rank)
    fd = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in fields.items()}
    cd = torch.from_numpy(depth.view(np.int32).copy()).to(dev)
    st = pygdf.path_state(fd, cd)
    box, px = pygdf.Aabb.of((-2.0, -1.0, -3.0), (4.0, 2.0, 1.0)), pygdf.TrainPixels(n_px, 0, 1)
    cap = n_px * 5
    ra, rb, rt = (torch.empty((cap, k), dtype=torch.float32, device=dev) for k in (9, 10, 9))
    for _ in range(args.warmup):
        n_rec = ctx.build_train_records(st, box, px, ra, rb, rt, stream=stream)
    rec_times = []
    for i in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        n_rec = ctx.build_train_records(st, box, px, ra, rb, rt, stream=stream)
        e.record(stream)
        e.synchronize()
        rec_times.append(s.elapsed_time(e))
    # bytes every producer must move once: cur_depth, the delta flags of the
    # visited vertices, the 84 B of fields of each non-delta vertex, and the
    # 112 B of each record written
    visit = np.arange(5)[:, None] < depth[None, :].astype(np.int64)
    nondelta = visit & (fields["delta"] == 0)
    rec_bytes = 4 * n_px + int(visit.sum()) + 84 * int(nondelta.sum()) + 112 * n_rec
    return rec_times, n_rec, rec_bytes


def max_over_ranks(values, dist, device):
    """Each timing's maximum over all ranks: one all-reduce, which every rank
    calls with the same number of values (a single process returns them)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def job_rate(units_per_rank, world, ms):
    """Whole-job throughput: the units all ranks processed (each rank runs
    the same replica workload) over the slowest rank's step time in ms."""
    return units_per_rank * world / (ms * 1e-3)


def _report(args, rank, world, dist, dev, n, cfg, params, times, e2e_times, train_times, rec_times,
            last, n_rec, rec_bytes, clk, nb, workload_name, threads, q_h, wi_h, guided_h, form_times,
            grouped, serving, pcie=None, refgpu=None, kern=None):
    import torch
    ms = statistics.mean(times)
    ms_feat = statistics.mean(t[0] for t in kern["stage_ms"])
    ms_fused = statistics.mean(t[1] for t in kern["stage_ms"])
    ms_e2e = statistics.mean(e2e_times) if e2e_times else float("nan")
    ms_train = statistics.mean(train_times) if train_times else float("nan")
    ms_rec = statistics.mean(rec_times) if rec_times else float("nan")
    ms, ms_e2e, ms_train, ms_rec, ms_feat, ms_fused = max_over_ranks(
        [ms, ms_e2e, ms_train, ms_rec, ms_feat, ms_fused], dist, dev)
    value = job_rate(n, world, ms)
    e2e_value = job_rate(n, world, ms_e2e)
    h2d = q_h.nbytes + wi_h.nbytes + guided_h.nbytes
    d2h = wi_h.nbytes

    if rank == 0:
        peaks = load_peaks()
        flops = FLOP_PER_QUERY[args.workload] * n
        achieved = flops / (ms * 1e-3) / 1e12  # average launch duration
        traffic, k_traffic = None, {}
        prof = os.path.join(ROOT, "profiles", f"infer_step_{args.workload}.json")
        if os.path.exists(prof):
            pj = json.load(open(prof))
            traffic = pj.get("dram_bytes_per_step")
            k_traffic = pj.get("dram_bytes", {})
        # per kernel, each against its own CUDA-event duration in this run
        fused_tf = flops / (ms_fused * 1e-3) / 1e12
        feat_bytes = FEATURE_BYTES_PER_QUERY[args.workload] * n + kern["grid_bytes"]
        feat_gbs = feat_bytes / (ms_feat * 1e-3) / 1e9
        kernels = [
            {"kernel": "df_fused_kernel", "bound": "tensor", "achieved": fused_tf, "peak": peaks["bf16_tflops"],
             "unit": "TFLOP/s", "frac": fused_tf / peaks["bf16_tflops"], "traffic": k_traffic.get("df_fused_kernel"),
             "ms": ms_fused, "algorithmic": f"{FLOP_PER_QUERY[args.workload]} flop per query (theta + phi MLPs)"},
            {"kernel": "grid_features_kernel", "bound": "hbm", "achieved": feat_gbs, "peak": peaks["hbm_gbs"],
             "unit": "GB/s", "frac": feat_gbs / peaks["hbm_gbs"], "traffic": k_traffic.get("grid_features_kernel"),
             "ms": ms_feat,
             "algorithmic": f"{FEATURE_BYTES_PER_QUERY[args.workload]} B per query (positions read, both "
                            f"networks' fp16 features written) + {kern['grid_bytes']} B of fp16 tables; its "
                            f"measured bound is the L1-to-L2 request rate of the random gathers, not HBM"},
        ]
        dominant = max(kernels, key=lambda k: k["ms"])
        if args.cpu_seconds > 0:
            cpu_v, cpu_n, cpu_s = cpu_sample(cfg, params, args.cpu_seconds, threads)
        else:
            cpu_v, cpu_n, cpu_s = None, 0, 0.0
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp16 (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": workload_name, "queries": n, "l2": "flushed (256 MiB) between steps",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
            "roofline": {**{k: dominant[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic",
                                                      "kernel", "ms")},
                         "peak_source": peaks["source"],
                         "dominant": "the longer of the step's two kernels in this run",
                         "kernels": kernels,
                         "step": {"kernels": "grid_features_kernel + df_fused_kernel", "achieved": achieved,
                                  "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"],
                                  "traffic": traffic}},
            "cpu_baseline": {"value": cpu_v, "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": f"{cpu_n} queries ({cpu_s:.1f} s): the bounce's first 131,072 queries "
                                       f"repeated; reference epilogue (train.h) compiled for the host after a "
                                       f"scalar fp32 forward of the same networks and weights"},
        }
        if train_times:
            line["train"] = {
                "metric": "train samples/s", "value": job_rate(nb, world, ms_train),
                "unit": "records/s", "batch": nb, "ms_per_step": ms_train,
                "achieved_tflops": TRAIN_FLOP_PER_RECORD[args.workload] * nb / (ms_train * 1e-3) / 1e12,
                "loss": last.loss, "launches_per_step": 10}
        if rec_times:
            line["records"] = {
                "metric": "training records/s (generate_training_data_AR)",
                "value": job_rate(n_rec, world, ms_rec), "unit": "records/s",
                "pixels": n, "records": n_rec, "ms_per_step": ms_rec, "algorithmic_bytes": rec_bytes,
                "achieved_gbs": rec_bytes / (ms_rec * 1e-3) / 1e9,
                "frac_hbm": rec_bytes / (ms_rec * 1e-3) / 1e9 / peaks["hbm_gbs"],
                "launches_per_step": 3}
        if pcie:
            # the copies alone, one direction after the other, at the box's
            # pinned-copy bandwidth; the step overlaps them with each other
            # and with the kernels, so its floor is the slower direction
            floor = max(h2d / (pcie["h2d_gbs"] * 1e9), d2h / (pcie["d2h_gbs"] * 1e9)) * 1e3
            line["e2e"].update({"pinned_copy_gbs": pcie, "copy_floor_ms": floor,
                                "frac_of_copy_floor": floor / ms_e2e})
        what = {"bf16": "bf16 MLP operands (fp32 accumulation)",
                "fp8": "e4m3 hidden matrices, per-matrix and per-row power-of-two scales (fp32 accumulation)"}
        for name, ts in form_times.items():
            if name == "bf16_train":
                continue
            mb = statistics.mean(ts)
            line[name] = {"metric": "guided queries/s, " + what[name],
                          "value": job_rate(n, world, mb), "unit": "queries/s", "ms_per_step": mb,
                          "vs_fp16": ms / mb}
        if "bf16_train" in form_times and "bf16" in line:
            mt = statistics.mean(form_times["bf16_train"])
            line["bf16"]["train"] = {"metric": "train samples/s, bf16 training form", "batch": nb,
                                     "value": job_rate(nb, world, mt), "unit": "records/s",
                                     "ms_per_step": mt, "vs_fp16": ms_train / mt if train_times else None}
        if refgpu:
            line["reference_gpu"] = refgpu
        if grouped:
            line["grouped"] = grouped
        if serving:
            line["serving"] = serving
        line.update({
            "clocks": clk,
            "gpu_launches": 2 * args.steps,  # grid features + fused kernel per step
        })
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
