#!/usr/bin/env python3
"""Particle-filter step throughput on B200 (particle-steps/s).

Default workload (N=1, --workload plain): the large unicycle filter -- 2^20
particles as 2048 sub-filters of 512 on a 32 x 64 torus, top-2 exchange with
each neighbour, systematic (--resampler vose: Vose alias) resampling every
step, FP32 state and log-weights, FP64 normalisation and cumulative sums,
seed 2, 1000 steps.  Inputs (controls and range/bearing measurements to 4
landmarks) are synthetic, generated from the seed.  A "step" is one full
filter step over all 2^20 particles.
--workload arm: the 6-joint DH arm, 2^18 particles = 1024 x 256 on a 32 x 32
torus, t = 1, seed 3.  --workload beacon: the reference unicycle program's
range-only model (10 beacons) at the plain workload's shape and seed.
--workload batched / served: the batched uneven
filters and the served tracking load (their own JSON lines).

value:  device-timed (CUDA events on the filter's stream), inputs resident
        in HBM, one CUDA-graph replay per step, L2 flushed (256 MB write)
        before every timed step.  value = particles * steps / sum(step time).
e2e:    the same through the public API with host inputs: pf_step_submit /
        pf_step_collect (pipelined; H2D of the 128-byte step input and D2H
        of the estimate for every step inside the timed region, the L2 flush
        time subtracted); e2e.sync: pf_step, one synchronous step at a time.
roofline: the dominant kernel's algorithmic bytes (the sampling kernel reads
        the state, 12 B per unicycle particle; the resampling kernel writes
        it) over its CUDA-event time, against the measured HBM copy
        bandwidth; `step` gives the whole step (24 B per particle-step).
        traffic: the kernel's DRAM bytes per launch from the committed ncu
        summary; issue: the same kernel against the instruction-issue
        roofline (its ncu warp-instruction count at 4 issues per cycle per
        SM at the sampled clock), the bound it actually meets.

clocks: nvidia-smi samples (20 ms) over a window of more than a second:
        untimed steps of the same work for ~0.8 s before and after the timed ones.
latency_ms: pf_step's per-step latency on the host (p50/p99/p999) beside the
        device step times.

Multi-GPU (torchrun): each rank runs its own filter (weak scaling, replicas,
no data-path collective); time = max over ranks.
--impl reference: the CPU restatement of the reference step (the reference's
OpenCL path cannot run here) on all host cores, on the full workload shape
(W warm-up steps, then the K timed steps in >= 3 repeats, time-bounded; the
median repeat); its inputs come from oracle/workload.py, so that process never
loads the engine.  The plain line's cpu_baseline is the same, bounded to 20 s.
"""
import argparse
import ctypes as C
import json
import os
import signal
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ALG_BYTES = 24  # unicycle, per particle-step
MAX_ROLL = 40000  # untimed steps at most on either side of the timed ones (clock window)
# single-filter workloads: model, sub-filter size, sub-filters, torus transfer,
# seed, algorithmic bytes per particle-step (state read + write)
WORKLOADS = {
    "plain": dict(model=0, m=512, nsub=2048, t=2, seed=2, alg=24, angles=(), torus=(32, 64),
                  desc="unicycle 2^20 particles = 2048 sub-filters x 512, torus 32x64, t=2"),
    "arm": dict(model=1, m=256, nsub=1024, t=1, seed=3, alg=96, angles=(0, 1, 2, 3, 4, 5), torus=(32, 32),
                desc="6-joint DH arm 2^18 particles = 1024 sub-filters x 256, torus 32x32, t=1"),
    "beacon": dict(model=3, m=512, nsub=2048, t=2, seed=2, alg=24, angles=(), torus=(32, 64),
                   desc="10-beacon range-only unicycle 2^20 particles = 2048 sub-filters x 512, torus 32x64, t=2"),
}
CONFIGS = {
    "systematic": 1,
    "vose": 2,
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 20 ms, read by a thread.
    start() returns once the first sample has arrived (the sampler takes a
    while to come up), so a window of load begun after it is covered."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.cmd = ["nvidia-smi", "-i", str(gpu_index),
                    "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                    "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                    "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                    "--format=csv,noheader,nounits", "-lms", "20"]
        self.lines, self.proc, self.thread = [], None, None
        self.t_start = self.t_stop = None

    def start(self, wait_s=10.0):
        import threading
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self

        def read():
            for line in self.proc.stdout:
                self.lines.append((time.perf_counter(), line))

        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()
        t0 = time.perf_counter()
        while not self.lines and time.perf_counter() - t0 < wait_s and self.proc.poll() is None:
            time.sleep(0.01)
        return self

    def mark(self, start):
        """Brackets the window whose samples are summarised (the load window)."""
        if start:
            self.t_start = time.perf_counter()
        else:
            self.t_stop = time.perf_counter()

    def stop(self):
        if self.proc is None:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, reasons, power = [], None, set(), []
        for t, line in self.lines:
            if self.t_start is not None and not (self.t_start <= t <= (self.t_stop or t)):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
                power.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(self.NAMES, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "window_s": (self.t_stop - self.t_start) if self.t_start and self.t_stop else None,
                "power_w_median": float(np.median(power)) if power else None}


def visible_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local_rank < len(ids):
            return ids[local_rank].strip()
    return str(local_rank)


def model_params(E, W):
    if W["model"] == 3:
        return E.beacon_params()
    return E.unicycle_params(W["seed"]) if W["model"] == 0 else E.dharm_params(W["seed"])


def workload_config(W, resampler_name, extra=None):
    """The `config` both arms report for a single-filter workload."""
    c = {"workload": "%s, %s resampling every step, FP32 state/log-weights, FP64 normalisation+cumsum"
                     % (W["desc"], resampler_name),
         "particles": W["m"] * W["nsub"], "subfilters": W["nsub"], "particles_per_subfilter": W["m"],
         "torus": W["torus"], "num_transfer": W["t"], "seed": W["seed"]}
    c.update(extra or {})
    return c


def cpu_filter_run(W, resampler, warmup, steps, budget_s, repeats=3):
    """The oracle's whole step (C, OpenMP over all host cores) on the full
    workload (same shape, torus, t and seeded trace as the GPU arm), built
    from oracle/workload.py so the process never loads the engine.  Runs
    `warmup` untimed steps, then up to `steps` timed steps split into
    `repeats` (>= 3) equal chunks, stopping early at `budget_s`; the value is
    the median chunk throughput."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    import workload as Wk
    m, nsub = W["m"], W["nsub"]
    p = Wk.params(W["model"], W["seed"])
    total = warmup + max(steps, repeats)
    control, meas, _, _ = Wk.make_trace(W["model"], p, W["seed"], total)
    md = O.model_from_params(W["model"], p)
    S = Wk.NUM_STATE[W["model"]]
    f = O.Filter(md, m, nsub, W["t"], O.EXCH_TORUS, resampler, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                 np.array(p.init_state[:S], np.float32))
    t_w = time.perf_counter()
    k = 0
    for k in range(max(warmup, 1)):
        f.step(control[k], meas[k])
        if time.perf_counter() - t_w > budget_s / 4:
            break
    step_s = (time.perf_counter() - t_w) / (k + 1)
    k += 1
    timed = max(repeats, min(steps, int(budget_s / max(step_s, 1e-6))))
    chunk = max(1, timed // repeats)
    rates = []
    for r in range(repeats):
        t0 = time.perf_counter()
        for _ in range(chunk):
            f.step(control[k % total], meas[k % total])
            k += 1
        rates.append(m * nsub * chunk / (time.perf_counter() - t0))
    f.close()
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    return {"value": float(np.median(rates)), "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "repeats": [float(x) for x in rates],
            "sample": "%d repeats x %d steps of the full workload (%s, torus %dx%d, t=%d); median of the repeats"
                      % (repeats, chunk, W["desc"].split(" = ")[0], W["torus"][0], W["torus"][1], W["t"]),
            "cpu": cpu_model()}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_arm(args, rank, world):
    """The reference's CPU path of the step: the oracle's C restatement (the
    reference's own OpenCL-on-CPU path cannot run on these hosts), full
    workload shape, all host cores; rank 0 only."""
    resampler = CONFIGS[args.resampler]
    if rank != 0:
        return 0
    W = WORKLOADS.get(args.workload, WORKLOADS["plain"])
    base = cpu_filter_run(W, resampler, args.warmup, args.steps, budget_s=150.0)
    line = {"metric": "particle-steps/s", "value": base["value"], "unit": "particle-steps/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded trace, seed %d)"
            % W["seed"], "config": workload_config(W, args.resampler),
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference's OpenCL-on-CPU path is not runnable (no CPU OpenCL runtime); this is the "
                    "oracle's C restatement of the reference step, OpenMP over sub-filters; inputs from "
                    "oracle/workload.py (the engine's library is not loaded)"}
    print(json.dumps(line), flush=True)
    return 0


def run_batched(E, torch, args, local):
    """Batched uneven filters: 4096 unicycle filters, counts log-uniform over
    [256, 65536] rounded to 256, 200 steps, one graph-captured launch per run;
    largest sub-filter size / particles per thread / threads per particle /
    exchange period picked by pf_batch_autotune on a 256-filter slice (each
    filter runs the largest sub-filter size up to the picked one that divides
    its count); compared with looping the plain single-filter path (pf_step per
    filter and step, each filter's own sub-filter size) over a sample of the
    same filters."""
    from esthera_b200 import workloads as W
    steps = args.batch_steps
    counts, params, inputs, truth = W.batched_unicycle(args.batch_filters, steps)
    F = len(counts)
    P = int(counts.sum())
    base = dict(num_transfer=2, exchange=E.EXCHANGE_RING, resampler=E.RESAMPLE_SYSTEMATIC, seed=4, device=local)
    # autotune on an evenly spaced slice of the filters, 16 steps
    sl = np.arange(0, F, max(1, F // 256))[:256]
    t0 = time.time()
    best, table = E.batch_autotune(E.MODEL_UNICYCLE, [params[i] for i in sl], counts[sl], inputs[sl, :16],
                                   truth[sl, :16], m_list=(128, 256, 512, 1024), ppt_list=(2, 4), tpp_list=(1, 2),
                                   period_list=(1, 2, 4), burn_in=4, rmse_tol=0.02, **base)
    tune_s = time.time() - t0
    cfg = dict(base, particles_per_subfilter=best.particles_per_subfilter,
               particles_per_thread=best.particles_per_thread, threads_per_particle=best.threads_per_particle,
               exchange_period=best.exchange_period)
    B = E.FilterBatch(E.MODEL_UNICYCLE, params, counts, **cfg)
    info = B.info()
    shapes = [B.filter_shape(f) for f in range(F)]
    offsets = [B.filter_info(f)["stream_offset"] for f in range(F)]
    d_in = torch.from_numpy(np.ascontiguousarray(inputs).view(np.uint8).reshape(-1).copy()).cuda()
    d_est = torch.zeros(F * steps * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(B.stream(), device=torch.device("cuda", local))
    init = np.stack([np.array(p.init_state[:3], np.float32) for p in params])
    # warm-up run (captures the graph), then the timed run from the initial states
    B.submit(d_in.data_ptr(), d_est.data_ptr(), steps, steps)
    B.synchronize()
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE).reshape(F, steps)  # from fresh streams
    B.set_initial_states(init)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    B.submit(d_in.data_ptr(), d_est.data_ptr(), steps, steps)
    ev1.record(stream)
    ev1.synchronize()
    run_ms = ev0.elapsed_time(ev1)
    err = est["mean"][:, :, :2] - truth[:, :, :2]
    rmse_f = np.sqrt(np.mean(np.sum(err[:, 20:] ** 2, axis=-1), axis=1))
    value = P * steps / (run_ms * 1e-3)
    # end to end through pf_batch_step: host inputs in, host estimates out, per step
    B.set_initial_states(init)
    lat = []
    e2e_steps = min(steps, args.batch_e2e_steps)
    for k in range(e2e_steps):
        ev0.record(stream)
        B.step(inputs[:, k])
        ev1.record(stream)
        ev1.synchronize()
        lat.append(ev0.elapsed_time(ev1))
    B.close()
    # plain path: one filter at a time through pf_step (each filter's own m and
    # ppt, the same period and streams, so the results are identical to the
    # batched ones)
    sample = np.arange(0, F, max(1, F // args.plain_sample))[:args.plain_sample]
    plain_s, plain_ps, same = 0.0, 0, True
    rest = {k: v for k, v in cfg.items() if k not in ("particles_per_subfilter", "particles_per_thread")}
    for mf, e in sorted(set(shapes)):  # load each kernel once; every sampled filter below starts fresh
        warm = E.ParticleFilter(E.MODEL_UNICYCLE, params[0], particles_per_subfilter=mf, particles_per_thread=e,
                                num_subfilters=1, pipeline=E.PIPELINE_SPLIT, **rest)
        warm.step(inputs[0, 0])
        warm.close()
    for i in sample:
        n = int(counts[i])
        mf, e = shapes[i]
        f = E.ParticleFilter(E.MODEL_UNICYCLE, params[i], particles_per_subfilter=mf, particles_per_thread=e,
                             num_subfilters=n // mf, pipeline=E.PIPELINE_SPLIT, stream_offset=int(offsets[i]),
                             **rest)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(steps):
            e = f.step(inputs[i, k])
        plain_s += time.perf_counter() - t0
        plain_ps += n * steps
        same = same and bool(np.array_equal(e["mean"], est[i, steps - 1]["mean"]))
        f.close()
    plain = plain_ps / plain_s
    lat = np.array(lat)
    return {
        "metric": "particle-steps/s (batched uneven filters)", "value": value, "unit": "particle-steps/s",
        "steps": steps, "ms_per_step": run_ms / steps, "higher_is_better": True,
        "config": {"workload": "%d unicycle filters, particle counts log-uniform [256, 65536] rounded to 256 "
                               "(total %d), landmarks from seed 4+i, ring exchange t=2, systematic resampling, "
                               "%d steps in one graph launch" % (F, P, steps),
                   "filters": F, "particles": P, "subfilters": info["total_subfilters"],
                   "particles_per_subfilter": cfg["particles_per_subfilter"],
                   "subfilter_sizes": {str(mf): int(sum(1 for s in shapes if s[0] == mf))
                                       for mf in sorted({s[0] for s in shapes})},
                   "particles_per_thread": cfg["particles_per_thread"],
                   "threads_per_particle": cfg["threads_per_particle"], "exchange_period": cfg["exchange_period"],
                   "l2": "working set %.1f GB > L2" % (info["device_bytes"] / 1e9)},
        "roofline": {"bound": "hbm", "achieved": ALG_BYTES * P * steps / (run_ms * 1e-3) / 1e9, "unit": "GB/s"},
        "e2e": {"value": P * e2e_steps / (lat.sum() * 1e-3), "unit": "particle-steps/s",
                "h2d_bytes_per_step": F * 128, "d2h_bytes_per_step": F * int(E.ESTIMATE_DTYPE.itemsize)},
        "latency_ms": {"what": "one step of all filters through pf_batch_step (host in/out)",
                       "p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "p999": float(np.percentile(lat, 99.9))},
        "plain_loop": {"value": plain, "unit": "particle-steps/s",
                       "sample": "%d filters x %d steps through pf_step, same configuration" % (len(sample), steps),
                       "identical_results": same, "speedup": value / plain},
        "rmse_xy": {"mean": float(rmse_f.mean()), "p99": float(np.percentile(rmse_f, 99))},
        "autotune": {"seconds": tune_s, "slice": "%d filters x 16 steps" % len(sl),
                     "candidates": [{"m": r["particles_per_subfilter"], "ppt": r["particles_per_thread"],
                                     "tpp": r["threads_per_particle"], "period": r["exchange_period"],
                                     "ms_per_step": r["ms_per_step"], "rmse": r["rmse"], "accepted": r["accepted"]}
                                    for r in table if r["status"] == 0],
                     "not_runnable": len([r for r in table if r["status"] != 0])},
        "gpu_launches": 3 * steps,
    }


def run_served(E, args, local):
    """Served tracking load: Poisson arrivals (2000 req/s), 70% unicycle / 30%
    DH arm, particle counts log-uniform over [1024, 262144] (rounded to m),
    50-500 updates per request spaced 1-20 ms, seed 5, 150 GB HBM budget; the
    C request loop (pf_serve_load) runs in real time with continuous batching."""
    cfg = E.default_config(particles_per_subfilter=256, particles_per_thread=4, num_transfer=2,
                           exchange=E.EXCHANGE_RING, resampler=E.RESAMPLE_SYSTEMATIC, device=local)
    rep = E.serve_load(cfg, rate=args.serve_rate, duration_s=args.serve_seconds)
    return {
        "metric": "particle-steps/s (served tracking load)", "value": rep["particle_steps_per_s"],
        "unit": "particle-steps/s", "higher_is_better": True,
        "config": {"workload": "Poisson %.0f req/s for %.0f s, 70%% unicycle / 30%% DH arm, particles log-uniform "
                               "[1024, 262144] rounded to 256, 50-500 updates 1-20 ms apart, seed 5, 150 GB budget"
                               % (args.serve_rate, args.serve_seconds),
                   "particles_per_subfilter": 256, "particles_per_thread": 4, "exchange": "ring t=2"},
        "latency_ms": {"p50": rep["lat_p50_ms"], "p99": rep["lat_p99_ms"], "p999": rep["lat_p999_ms"],
                       "max": rep["lat_max_ms"], "what": "measurement due -> estimate on the host"},
        "demanded_particle_steps_per_s": rep["demanded_particle_steps_per_s"],
        "report": rep,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--resampler", default="systematic", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--phase-steps", type=int, default=100, help="steps of the per-kernel timing pass")
    ap.add_argument("--ppt", type=int, default=0,
                    help="particles per thread (split pipeline; 0: the library's default for the model and m)")
    ap.add_argument("--pipeline", default="split", choices=["fused", "split"])
    ap.add_argument("--workload", default="plain", choices=["plain", "arm", "beacon", "batched", "served"])
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--batch-filters", type=int, default=4096)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--batch-e2e-steps", type=int, default=50)
    ap.add_argument("--plain-sample", type=int, default=64)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    import esthera_b200 as E
    if args.workload == "batched":
        if rank == 0 or world == 1:
            line = run_batched(E, torch, args, local)
            line.update({"n_gpus": 1, "warmup": 1, "scaling": "none", "vs_baseline": None, "dtype": "f32",
                         "data": "synthetic (seeded traces, seeds 4+i)"})
            peak, kind = peaks()
            line["roofline"].update({"peak": peak, "frac": line["roofline"]["achieved"] / peak, "peak_kind": kind})
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "served":
        if rank == 0 or world == 1:
            line = run_served(E, args, local)
            line.update({"n_gpus": 1, "scaling": "none", "vs_baseline": None, "dtype": "f32",
                         "data": "synthetic (seeded requests, seed 5)"})
            print(json.dumps(line), flush=True)
        return 0
    resampler = CONFIGS[args.resampler]
    W = WORKLOADS[args.workload]
    m, nsub, particles = W["m"], W["nsub"], W["m"] * W["nsub"]
    p = model_params(E, W)
    # the trace covers warm-up, the clock window's untimed steps before and
    # after the timed ones (at most MAX_ROLL each) and the timed steps
    total_steps = args.warmup + args.steps + 2 * MAX_ROLL
    inputs, truth = E.make_trace(W["model"], p, W["seed"], total_steps)
    f = E.ParticleFilter(W["model"], p, particles_per_subfilter=m, num_subfilters=nsub, num_transfer=W["t"],
                         exchange=E.EXCHANGE_TORUS, resampler=resampler, seed=W["seed"] + 1000 * rank, device=local,
                         particles_per_thread=args.ppt if args.pipeline == "split" else 0,
                         pipeline={"fused": E.PIPELINE_FUSED, "split": E.PIPELINE_SPLIT}[args.pipeline])
    info = f.info()
    stream = torch.cuda.ExternalStream(f.stream(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    d_in = torch.from_numpy(inputs[:total_steps].view(np.uint8).copy()).cuda()
    d_est = torch.zeros(total_steps * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    # warm-up: builds the graph and runs W steps (no per-launch events in the timed graph)
    t_w = time.perf_counter()
    f.run_device(d_in.data_ptr(), d_est.data_ptr(), total_steps, 1)
    f.synchronize()
    t_w = time.perf_counter()
    for k in range(args.warmup - 1):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        f.run_continue(1)
    f.synchronize()
    per_step_s = (time.perf_counter() - t_w) / max(args.warmup - 1, 1)
    # the clock window: untimed steps (same work, same L2 flush) for about
    # 0.8 s before and after the timed steps, so the nvidia-smi samples
    # (every 20 ms) cover more than a second of this load around them
    roll = int(min(MAX_ROLL, max(1, np.ceil(0.8 / max(per_step_s, 1e-6)))))

    def untimed(n):
        for k in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            f.run_continue(1)
        f.synchronize()

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(visible_gpu_index(local)).start() if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clk:
        clk.mark(True)
    untimed(roll)
    step_ms, phase_ms = [], {}
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            ev0.record(stream)
        f.run_continue(1)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    untimed(roll)
    if clk:
        clk.mark(False)
    if dist:
        dist.barrier()
    clocks = clk.stop() if clk else None
    steps_run = args.warmup + 2 * roll + args.steps
    total_ms = float(np.sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE)
    value = world * particles * args.steps / (total_ms * 1e-3)

    # per-kernel times: a separate pass with an event recorded around every
    # launch (event nodes in the graph), same L2 flush before each step; the
    # pass replays the trace from its start, so the particles restart from the
    # initial state (the Vose build's cost depends on the weights)
    f.set_initial_state(np.array(p.init_state[:E.model_info(W["model"])[0]], np.float32))
    f.set_timing(True)
    f.run_device(d_in.data_ptr(), d_est.data_ptr(), total_steps, 1)
    f.synchronize()
    for k in range(args.phase_steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        f.run_continue(1)
        for name, ms in f.last_step_timing():
            phase_ms.setdefault(name, []).append(ms)
    f.set_timing(False)
    # one untimed submit / collect: it captures the step graph over the pinned
    # rings (set-up done once per filter, like the device run's warm-up)
    f.submit(E.step_input(inputs[0]))
    f.collect()
    f.set_initial_state(np.array(p.init_state[:E.model_info(W["model"])[0]], np.float32))

    # end to end through the public API, pipelined: pf_step_submit (host input
    # -> pinned ring -> H2D on an upload stream, the step graph waiting for it)
    # and pf_step_collect (estimate D2H on a download stream into a pinned
    # ring).  L2 is flushed before every step on the filter's stream; the
    # flushes carry events of their own and their time is subtracted.
    K = args.e2e_steps
    fl = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    step_in = [E.step_input(inputs[k]) for k in range(K)]  # the host inputs, as a caller holds them
    got = []
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for k in range(K):
            fl[k][0].record(stream)
            flush.fill_(float(k))
            fl[k][1].record(stream)
            if k - len(got) >= E.QUEUE_DEPTH:  # ring full: wait for the oldest step
                got += list(f.collect(1))
            f.submit(step_in[k])  # from the initial state again, the trace from its start
            if k % 8 == 7:
                got += list(f.collect(wait=False))
        got += list(f.collect())
        ev1.record(stream)
    ev1.synchronize()
    assert len(got) == K and all(int(g["step"]) == k + 1 for k, g in enumerate(got))
    e2e_total = ev0.elapsed_time(ev1) - float(sum(a.elapsed_time(b) for a, b in fl))
    if dist:
        t = torch.tensor([e2e_total], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())

    # the synchronous call, one step at a time (the step latency a caller of pf_step sees)
    f.set_initial_state(np.array(p.init_state[:E.model_info(W["model"])[0]], np.float32))
    sync_ms, lat_ms = [], []
    for k in range(K):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            ev0.record(stream)
        stream.synchronize()  # the flush is done: the host clock below sees pf_step alone
        t0 = time.perf_counter()
        f.step(inputs[k])
        lat_ms.append((time.perf_counter() - t0) * 1e3)
        ev1.record(stream)
        ev1.synchronize()
        sync_ms.append(ev0.elapsed_time(ev1))
    sync_total = float(np.sum(sync_ms))
    if dist:
        t = torch.tensor([sync_total], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sync_total = float(t.item())
    e2e_value = world * particles * args.e2e_steps / (e2e_total * 1e-3) if args.e2e_steps > 0 else None

    if rank == 0:
        peak, peak_kind = peaks()
        mean_step_ms = total_ms / args.steps
        phases = {n: float(np.mean(v)) for n, v in phase_ms.items()}
        dom = max(phases, key=phases.get)
        # algorithmic bytes per particle by kernel: the sampling kernel reads the
        # state (12 B), the resampling kernel writes it (12 B), the single-kernel
        # step does both
        alg = W["alg"]
        kernel_alg = {"sample_sort": alg // 2, "exchange_resample": alg // 2, "step": alg}.get(dom, alg)
        achieved = kernel_alg * particles / (phases[dom] * 1e-3) / 1e9
        step_achieved = alg * particles / (float(np.mean(step_ms)) * 1e-3) / 1e9
        traffic, prof = None, {}
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists():
            prof = json.loads(tp.read_text()).get("%s %s ppt%d" % (args.workload, args.pipeline,
                                                                   info["particles_per_thread"]), {})
            traffic = prof.get(dom, {}).get("dram_bytes_per_launch")
        # the issue roofline the kernels are actually bound by: warp instructions
        # per launch (ncu, profiles/) over 4 issues per cycle per SM at the
        # sampled SM clock
        issue = None
        winst = prof.get(dom, {}).get("warp_instructions_per_launch")
        if winst and clocks and clocks.get("sm_mhz"):
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            min_ms = winst / (4.0 * sms * clocks["sm_mhz"] * 1e6) * 1e3
            issue = {"warp_instructions_per_launch": winst, "min_ms_at_full_issue": min_ms,
                     "frac": min_ms / phases[dom], "sms": sms, "sm_mhz": clocks["sm_mhz"]}
        if W["angles"]:  # joint angles, wrapped
            d = est["mean"][:steps_run, list(W["angles"])] - truth[:steps_run, list(W["angles"])]
            d = np.remainder(d + np.pi, 2 * np.pi) - np.pi
        else:  # position
            d = est["mean"][:steps_run, :2] - truth[:steps_run, :2]
        rmse = float(np.sqrt(np.mean(np.sum(d ** 2, axis=1))))
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded trace, seed %d)" % W["seed"],
            "config": workload_config(W, args.resampler, {
                "particles_per_thread": info["particles_per_thread"], "rng": "MTGP32 per sub-filter",
                "pipeline": {0: "fused (one kernel per step)", 1: "phased", 2: "split"}[info["pipeline"]],
                "l2": "flushed before every timed step (256 MB write)",
                "parallelism": "replicas" if world > 1 else "single GPU"}),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "kernel": dom, "kernel_ms": phases[dom], "share": phases[dom] / sum(phases.values()),
                         "alg_bytes_per_launch": kernel_alg * particles,
                         "ncu": prof.get(dom, {}).get("summary"), "issue": issue,
                         "step": {"achieved": step_achieved, "frac": step_achieved / peak,
                                  "alg_bytes_per_particle_step": alg, "phase_ms": phases}},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 128,
                    "d2h_bytes_per_step": int(E.ESTIMATE_DTYPE.itemsize),
                    "ms_per_step": e2e_total / args.e2e_steps if args.e2e_steps > 0 else None,
                    "api": "pf_step_submit + pf_step_collect (pipelined, %d steps; L2 flush time subtracted)"
                           % args.e2e_steps,
                    "sync": {"value": world * particles * args.e2e_steps / (sync_total * 1e-3)
                             if args.e2e_steps > 0 else None, "ms_per_step": sync_total / max(args.e2e_steps, 1),
                             "api": "pf_step (synchronous, one step at a time)"}},
            "latency_ms": {"what": "pf_step (synchronous, host input -> estimate on the host), one step at a "
                                   "time from an idle GPU with L2 flushed, %d steps" % K,
                           "p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                           "p999": float(np.percentile(lat_ms, 99.9)),
                           "device_step": {"what": "timed steps, CUDA events around each graph launch",
                                           "p50": float(np.percentile(step_ms, 50)),
                                           "p99": float(np.percentile(step_ms, 99))}},
            "gpu_launches": int(args.steps * len(phases)),
            "timing": "value: CUDA events around each step's graph launch (no events inside); kernel times: "
                      "a separate %d-step pass with events between the launches" % args.phase_steps,
            "clocks": clocks,
            "rmse": {"value": rmse, "of": "joint angles (rad)" if W["angles"] else "x, y position (m)",
                     "steps": steps_run},
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_filter_run(W, resampler, 1, 1000, budget_s=20.0)
        print(json.dumps(line), flush=True)
    f.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
