#!/usr/bin/env python
"""Throughput benchmark: 2D type-1 + type-2 NUFFT, complex64, eps = 1e-6, 512 x 512 modes.

Workload (one step = one type-1 and one type-2 transform of each point set):
  (a) radial: 512 spokes x 1024 samples (M = 524,288), golden-angle spoke angles
      theta_s = s * pi (sqrt(5) - 1) / 2 mod pi, every radius uniform in [-pi, pi);
  (b) clustered: M = 4,000,000 points, x, y ~ N(0, 0.3^2) wrapped to [-pi, pi);
  strengths c and modes f iid complex N(0, 1); seeded synthetic data.
Metric: NU points per second, counting M once per transform (2 * (Ma + Mb) per step).

`value` times the steps with inputs resident in HBM (CUDA events, L2 flushed
between steps by writing a 256 MB buffer outside the timed events); the four
transforms of a step run on four CUDA streams (a type 2's deconvolve-pad and FFT
overlap the sort of its points), so their work overlaps.  `e2e` times
the same steps through the public API with pinned host buffers: host->device
copies of x, y, c, f and device->host copies of the results are inside the
timed region; uploads, compute and downloads run on separate streams so they
overlap: all uploads are queued first in the order the work needs them (x, y, f
of each set, then c), the type 2 runs first and its result downloads while c
uploads; consecutive steps are pipelined (a step's uploads run while the
previous step computes), and the timed region spans all K steps.
Inside the timed loop only the dominant kernel's library calls are bracketed
with CUDA events (its live launch time for `roofline`); the per-call breakdown
and the launch count come from one recorded warm-up step.
`cpu_baseline` times the CPU restatement of nufftax's pure-JAX path (oracle/)
on one core over one full step, and `accuracy` checks that step's GPU outputs
against it and against the FP64 direct sum on a subsample.  `--impl reference`
times the same restatement on all host cores on a bounded sample of each step.
Multi-GPU runs are independent replicas (weak scaling), timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
EPS = 1e-6
N_MODES = (512, 512)
METRIC = "type-1/2 NU points/s at eps 1e-6 (2D, 512^2 modes, complex64)"


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------
def radial_points(rng, n_spokes=512, n_samples=1024):
    """Radial trajectory: golden-angle spoke angles theta_s = s pi (sqrt(5) - 1) / 2
    mod pi, every sample's signed radius drawn uniform in [-pi, pi)."""
    ga = np.pi * (np.sqrt(5.0) - 1.0) / 2.0
    theta = np.mod(np.arange(n_spokes) * ga, np.pi)
    r = rng.uniform(-np.pi, np.pi, (n_spokes, n_samples))
    x = (r * np.cos(theta)[:, None]).ravel()
    y = (r * np.sin(theta)[:, None]).ravel()
    return x.astype(np.float32), y.astype(np.float32)


def clustered_points(M, rng, sigma=0.3):
    xy = sigma * rng.standard_normal((2, M))
    xy = np.mod(xy + np.pi, 2 * np.pi) - np.pi
    return xy[0].astype(np.float32), xy[1].astype(np.float32)


def workload(seed=1234, scale=1.0):
    rng = np.random.default_rng(seed)
    xa, ya = radial_points(rng, max(1, int(512 * scale)), 1024)
    Mb = max(1, int(4_000_000 * scale))
    xb, yb = clustered_points(Mb, rng)
    sets = []
    for name, x, y in (("radial", xa, ya), ("clustered", xb, yb)):
        M = x.size
        c = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
        f = (rng.standard_normal((N_MODES[1], N_MODES[0])) + 1j * rng.standard_normal(
            (N_MODES[1], N_MODES[0]))).astype(np.complex64)
        sets.append({"name": name, "x": x, "y": y, "c": c, "f": f, "M": M})
    return sets


DATA = ("synthetic (seeded): radial 512 golden-angle spokes x 1024 samples, radius uniform in [-pi, pi); "
        "4M points clustered N(0, 0.3^2) wrapped to [-pi, pi); c, f iid complex N(0, 1)")


def bench_config(world: int, sets) -> dict:
    """The workload the headline line (and the reference arm) is quoted on."""
    return {"workload": "2D type-1 + type-2, 512x512 modes, nf 1024x1024, eps 1e-6, ns 8: radial M=524288 and "
                        "clustered M=4000000 per step",
            "global_batch": points_per_step(sets) * world, "parallelism": f"replicas x{world}",
            "l2": "flushed between steps (256 MB write)",
            "sort": "every step: one sort per point set, shared by its type 1 and type 2"}


def points_per_step(sets):
    return sum(2 * s["M"] for s in sets)


# ---------------------------------------------------------------------------
# Environment helpers
# ---------------------------------------------------------------------------
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi takes a moment to start: wait (3 s at most) for its first
        # sample so that the samples cover the region that follows
        t0 = time.perf_counter()
        while not self.rows and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except ValueError:
                continue
            for n, v in zip(names, r[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def warm(step, n_min: int, seconds: float = 1.0) -> int:
    """Runs `step` at least n_min times and until `seconds` have passed (device
    synchronised), so that clock samples taken from here on see the GPU under
    this load.  Returns the number of steps run."""
    import torch

    n, t0 = 0, time.perf_counter()
    while n < n_min or time.perf_counter() - t0 < seconds:
        step()
        torch.cuda.synchronize()
        n += 1
    return n


class clocked:
    """`with clocked(index) as ck: ...` samples the SM clocks and throttle
    reasons while the block runs; ck.summary afterwards."""

    def __init__(self, index: int):
        self.sampler = ClockSampler(index)
        self.summary = None

    def __enter__(self):
        self.sampler.start()
        return self

    def __exit__(self, *exc):
        self.summary = self.sampler.stop()
        return False


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def aggregate_ranks(local_ms: float, points_per_rank: int, world: int, device) -> tuple[float, float]:
    """Replica timing across ranks: the job takes as long as the slowest rank
    (max over ranks of the device time) and processes every rank's points.
    Returns (max_ms, whole-job points per second)."""
    import torch

    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([float(local_ms)], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        local_ms = float(t.item())
    return local_ms, points_per_rank * world / (local_ms / 1e3)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
ALG_BYTES = {
    # algorithmic bytes per launch (complex64, d = 2): coordinates + strengths once, grid once
    "nfx_spread_sorted": lambda M, nf, nm: M * (4 * 2 + 8) + 8 * nf[0] * nf[1],
    "nfx_interp_sorted": lambda M, nf, nm: M * (4 * 2 + 8) + 8 * nf[0] * nf[1],
    "nfx_sort_points": lambda M, nf, nm: M * (4 * 2 + 4),
    "nfx_deconv_shuffle": lambda M, nf, nm: 16 * nm[0] * nm[1],
    "nfx_deconv_pad": lambda M, nf, nm: 8 * nm[0] * nm[1] + 8 * nf[0] * nf[1],
}


# Per-launch counters of the spread / interp kernels on each point set, from
# single-step ncu --metrics captures of `bench.py --case radial|clustered --reps 1`
# (profiles/k_spread_interp_2d_counters.md): DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum, caches flushed before the launch), warp instructions
# (smsp__inst_executed.sum) and shared-memory wavefronts
# (l1tex__data_pipe_lsu_wavefronts_mem_shared.sum).  The counts do not depend on
# timing, so the bench divides them by the live launch times to get the
# fractions of the issue and shared-memory roofs, the ones that bind these
# kernels (HBM runs at a few percent of peak).
MEASURED_COUNTERS = {
    "nfx_spread_sorted": {"radial": {"dram": 17.26e6, "inst": 40.75e6, "smem_wf": 6.39e6},
                          "clustered": {"dram": 84.82e6, "inst": 78.85e6, "smem_wf": 17.55e6}},
    "nfx_interp_sorted": {"radial": {"dram": 13.53e6, "inst": 7.31e6, "smem_wf": 3.71e6},
                          "clustered": {"dram": 102.01e6, "inst": 43.48e6, "smem_wf": 10.11e6}},
}
N_SMS = 148
ISSUE_PER_SM_CLK = 4      # one warp instruction per scheduler per clock, 4 schedulers per SM
SMEM_BYTES_PER_SM_CLK = 128  # one 128-byte shared-memory wavefront per SM per clock


def secondary_roofs(kernel: str, avg_launch_ms: float, sm_mhz) -> dict | None:
    """Fractions of the issue-slot and shared-memory-bandwidth roofs reached by the
    live launches of `kernel` (captured counts per launch / live launch time, against
    the SM count x per-clock rate x the median SM clock sampled in the run)."""
    counts = MEASURED_COUNTERS.get(kernel)
    if counts is None or not sm_mhz or avg_launch_ms <= 0:
        return None
    n = len(counts)
    inst = sum(c["inst"] for c in counts.values()) / n
    wf = sum(c["smem_wf"] for c in counts.values()) / n
    t = avg_launch_ms / 1e3
    clk = float(sm_mhz) * 1e6
    issue_peak = N_SMS * ISSUE_PER_SM_CLK * clk / 1e9
    smem_peak = N_SMS * SMEM_BYTES_PER_SM_CLK * clk / 1e9
    return {
        "issue": {"achieved": inst / t / 1e9, "peak": issue_peak, "unit": "G warp-instr/s",
                  "frac": inst / t / 1e9 / issue_peak, "inst_per_launch": inst},
        "shared": {"achieved": wf * 128 / t / 1e9, "peak": smem_peak, "unit": "GB/s",
                   "frac": wf * 128 / t / 1e9 / smem_peak, "wavefronts_per_launch": wf},
        "clock_mhz": float(sm_mhz),
        "counts_from": "ncu --metrics, one launch per point set (profiles/k_spread_interp_2d_counters.md)",
    }


def run_gpu(args):
    import torch

    import nufftax_b200 as nb
    from nufftax_b200 import profiling

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sets = workload(seed=1234 + rank)
    host = []
    for s in sets:
        h = {k: torch.from_numpy(s[k]).pin_memory() for k in ("x", "y", "c", "f")}
        h["M"] = s["M"]
        h["name"] = s["name"]
        host.append(h)
    devsets = [{k: (v.to(dev) if isinstance(v, torch.Tensor) else v) for k, v in h.items()} for h in host]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    kp = nb.compute_kernel_params(EPS)
    nf = tuple(nb.compute_grid_size(n, 2.0, kp.nspread) for n in N_MODES)

    # Each transform runs on its own stream: the type 1 of a point set (sort,
    # spread, FFT, deconvolution) on one, its type 2 on another, where the
    # deconvolve-pad and FFT run while the points sort and the interpolation
    # waits for the sort the type 1 made (the library's sort cache: an event
    # dependency).  The step is the union of the four, forked from and joined
    # to the main stream.
    main = torch.cuda.current_stream(dev)
    set_streams = [torch.cuda.Stream(dev) for _ in sets]
    t2_streams = [torch.cuda.Stream(dev) for _ in sets]

    def step(ds):
        # forked from and joined to the current stream (the capture stream while
        # a graph of the step is captured)
        cur = torch.cuda.current_stream(dev)
        nb.sort_cache.clear()
        outs = []
        for s, st, st2 in zip(ds, set_streams, t2_streams):
            st.wait_stream(cur)
            st2.wait_stream(cur)
            with torch.cuda.stream(st):
                f1 = nb.nufft2d1(s["x"], s["y"], s["c"], N_MODES, eps=EPS)
            with torch.cuda.stream(st2):
                c2 = nb.nufft2d2(s["x"], s["y"], s["f"], eps=EPS)
            outs.append((f1, c2))
        for st in set_streams + t2_streams:
            cur.wait_stream(st)
        return outs

    # The clock sampler (200 ms period) runs from the warm-up through the timed
    # region; warm-up continues past W steps until it has lasted 1 s so that the
    # samples reflect the clocks under this load.
    sampler = ClockSampler(local)
    sampler.start()
    t_w = time.perf_counter()
    n_w = 0
    while n_w < args.warmup or time.perf_counter() - t_w < 1.0:
        step(devsets)
        torch.cuda.synchronize()
        n_w += 1

    # One more warm-up step with CUDA events around every library call: the
    # per-call breakdown, the kernel launches of a step and the dominant single
    # kernel (the events cost host time, so the timed loop records only that one).
    with profiling.record() as rec0:
        step(devsets)
    torch.cuda.synchronize()
    per_call = rec0.summary()
    launches = sum(v["launches"] for v in per_call.values()) * args.steps
    ours = {k: v for k, v in per_call.items() if k in ALG_BYTES and k != "nfx_sort_points"}
    dom = max(ours, key=lambda k: ours[k]["ms"])
    breakdown = {k: {"calls": v["calls"], "ms_per_step": v["ms"]} for k, v in per_call.items()}

    # ---- timed region: device-resident inputs ---------------------------------
    # The step is captured once through the public API into a CUDA graph (the
    # analogue of the reference's jax.jit: the same kernels, sort included, with
    # no host work per launch) and replayed once per timed step; the dominant
    # kernel's calls are bracketed by event nodes inside the graph.  The eager
    # loop (host-bound: Python enqueues a step in about the device time) is
    # timed as well and reported beside it.
    stream = torch.cuda.current_stream(dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with profiling.record(only=[dom]) as rec_e:
        for i in range(args.steps):
            flush.fill_(float(i))
            starts[i].record(stream)
            step(devsets)
            ends[i].record(stream)
    torch.cuda.synchronize()
    eager_ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends)))
    eager_dom = rec_e.summary()[dom]

    graph = torch.cuda.CUDAGraph()
    with profiling.record(only=[dom]) as rec_g:
        with torch.cuda.graph(graph):
            graph_out = step(devsets)
    graph_dom_events = [(a, b) for name, a, b, _ in rec_g.events if name == dom]
    for _ in range(max(3, args.warmup)):
        graph.replay()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms, dom_ms = [], 0.0
    for i in range(args.steps):
        flush.fill_(float(i))
        starts[i].record(stream)
        graph.replay()
        ends[i].record(stream)
        # the event nodes are re-recorded by every replay: read them before the next
        ends[i].synchronize()
        step_ms.append(starts[i].elapsed_time(ends[i]))
        dom_ms += sum(a.elapsed_time(b) for a, b in graph_dom_events)
    total_ms = float(sum(step_ms))
    total_ms, value = aggregate_ranks(total_ms, points_per_step(sets) * args.steps, world, dev)
    pts = points_per_step(sets) * args.steps * world

    # roofline of the dominant single kernel, its launches timed live in the replays
    peak, peak_kind = measured_peaks()
    # every step launches the dominant kernel once per point set
    alg_total = args.steps * sum(ALG_BYTES[dom](s["M"], nf, N_MODES) for s in sets)
    n_dom = args.steps * len(graph_dom_events)
    alg_per_launch = alg_total / max(n_dom, 1)
    avg_ms = dom_ms / max(n_dom, 1)
    achieved = alg_total / (dom_ms / 1e3) / 1e9

    # ---- e2e: public API with pinned host buffers -------------------------------
    out_host = []
    for h in host:
        out_host.append((torch.empty((N_MODES[1], N_MODES[0]), dtype=torch.complex64).pin_memory(),
                         torch.empty(h["M"], dtype=torch.complex64).pin_memory()))
    h2d = sum(h[k].numel() * h[k].element_size() for h in host for k in ("x", "y", "c", "f"))
    d2h = sum(a.numel() * a.element_size() + b.numel() * b.element_size() for a, b in out_host)

    # Copies are served roughly in the order they are queued, so every upload is
    # queued first, on one upload stream, in the order the work needs them:
    # each set's x, y, f (the type 2 and the sort), then each set's c (the
    # type 1).  Each set computes on its own stream and downloads on its own
    # stream; the type 2 result downloads while the c uploads are still running
    # (PCIe is full duplex), and the type 1 reuses the sorted points.
    up = torch.cuda.Stream(dev)
    down_streams = [torch.cuda.Stream(dev) for _ in sets]
    # Two sets of device input buffers, used by alternate steps, as a pipelined
    # caller would keep them: a step's uploads go into a set only after the
    # transforms that read it two steps earlier are done (events), and no
    # device memory is allocated for inputs inside the timed loop.
    n_buf = 2
    dev_bufs = [[{k: torch.empty(h[k].shape, dtype=h[k].dtype, device=dev) for k in ("x", "y", "f", "c")}
                 for h in host] for _ in range(n_buf)]
    buf_free = [[] for _ in range(n_buf)]
    step_no = [0]

    def e2e_step():
        # no wait on the previous step: a step's uploads queue behind the
        # previous step's uploads on `up` and overlap its compute and downloads
        nb.sort_cache.clear()
        bi = step_no[0] % n_buf
        step_no[0] += 1
        for ev in buf_free[bi]:
            up.wait_event(ev)
        bufs = dev_bufs[bi]
        xyf_ev, c_ev = [], []
        with torch.cuda.stream(up):
            for h, d in zip(host, bufs):
                for k in ("x", "y", "f"):
                    d[k].copy_(h[k], non_blocking=True)
                xyf_ev.append(torch.cuda.Event())
                xyf_ev[-1].record(up)
            for h, d in zip(host, bufs):
                d["c"].copy_(h["c"], non_blocking=True)
                c_ev.append(torch.cuda.Event())
                c_ev[-1].record(up)
        live, done = [], []
        for d, (fo, co), st, down, xyf, cin in zip(bufs, out_host, set_streams, down_streams, xyf_ev, c_ev):
            x, y, f, c = d["x"], d["y"], d["f"], d["c"]
            st.wait_event(xyf)
            with torch.cuda.stream(st):
                c2 = nb.nufft2d2(x, y, f, eps=EPS)
                t2done = torch.cuda.Event()
                t2done.record(st)
            down.wait_event(t2done)
            with torch.cuda.stream(down):
                co.copy_(c2, non_blocking=True)
            c2.record_stream(down)
            st.wait_event(cin)
            with torch.cuda.stream(st):
                f1 = nb.nufft2d1(x, y, c, N_MODES, eps=EPS)
                t1done = torch.cuda.Event()
                t1done.record(st)
            down.wait_event(t1done)
            with torch.cuda.stream(down):
                fo.copy_(f1, non_blocking=True)
            f1.record_stream(down)
            done.append(t1done)
            live.append((c2, f1))
        buf_free[bi] = done
        return live

    def join_all():
        for s_ in [up] + set_streams + down_streams:
            main.wait_stream(s_)

    # warm-up pipelined like the timed loop, so the allocator already holds the
    # blocks that several steps in flight need
    for _ in range(max(5, args.warmup)):
        e2e_step()
    join_all()
    torch.cuda.synchronize()
    # K consecutive steps, pipelined: step i+1's uploads run while step i
    # computes and downloads; the timed region spans all of them (every step's
    # uploads and downloads inside it) and ends when the last download is done.
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for s_ in [up] + set_streams + down_streams:
        s_.wait_stream(main)
    for i in range(args.steps):
        e2e_step()
    join_all()
    b.record(stream)
    torch.cuda.synchronize()
    e_ms = a.elapsed_time(b)
    clocks = sampler.stop()
    e_ms, e2e_value = aggregate_ranks(e_ms, points_per_step(sets) * args.steps, world, dev)
    counters = MEASURED_COUNTERS.get(dom)
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (sum(c["dram"] for c in counters.values()) / len(counters) if counters else None),
                "traffic_note": "mean per launch over the two point sets, ncu capture with caches flushed",
                "alg_bytes_per_launch": alg_per_launch, "avg_launch_ms": avg_ms}
    sec = secondary_roofs(dom, avg_ms, clocks.get("sm_mhz"))
    if sec is not None:
        roofline["secondary"] = sec
        roofline["binding"] = max(("hbm", achieved / peak), ("issue", sec["issue"]["frac"]),
                                  ("shared", sec["shared"]["frac"]), key=lambda kv: kv[1])[0]

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "NU points/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "timing": "each step one replay of a CUDA graph captured through the public API (sort, spread, FFT, "
                  "deconvolution and interpolation kernels of both point sets); eager_* = the same steps "
                  "launched from Python",
        "eager_ms_per_step": eager_ms / args.steps,
        "eager_value": points_per_step(sets) * args.steps / (eager_ms / 1e3),
        "eager_dom_avg_launch_ms": eager_dom["ms"] / max(eager_dom["calls"], 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64",
        "data": DATA,
        "config": bench_config(world, sets),
        "e2e": {"value": e2e_value, "unit": "NU points/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps_pipelined": True,
                "pcie_gbs": round((h2d + d2h) * args.steps / (e_ms / 1e3) / 1e9, 1)},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "breakdown": breakdown,
    }
    if world == 1 and not args.no_subconfigs:
        # the other BASELINE configurations, measured in the same run (each with
        # its own clock record): 1D, the 64-problem batched mix, the
        # differentiated 3D step and a served mixed stream
        line["configs"] = {"plain_1d": measure_1d(dev, 50, 5),
                           "batched": measure_batched(dev, 10, 3, autotune=True),
                           "grad3d": measure_grad3d(dev, 5, 3),
                           "served": measure_serve(dev, args.served_requests, 300, [1.0, 4.0])}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # GPU results of one step at full size (the compute path of the timed
        # steps), checked in the CPU leg below against the oracle and the FP64
        # direct sum
        gpu_out = []
        for s in devsets:
            nb.sort_cache.clear()
            f1 = nb.nufft2d1(s["x"], s["y"], s["c"], N_MODES, eps=EPS)
            c2 = nb.nufft2d2(s["x"], s["y"], s["f"], eps=EPS)
            gpu_out.append((f1.cpu().numpy(), c2.cpu().numpy()))
        line["cpu_baseline"], line["accuracy"] = cpu_leg(sets, gpu_out)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# CPU legs: the oracle (restatement of nufftax's pure-JAX path)
# ---------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, str(ROOT))
    from oracle import nufft_oracle as O

    return O


def cpu_leg(sets, gpu_out):
    """The CPU leg of the headline run (rank 0, one GPU): the oracle (NumPy
    restatement of nufftax's pure-JAX path) runs one full step of the workload
    on one core, which is timed as `cpu_baseline`; its outputs, and the FP64
    direct sum on a subsample, then check the GPU's outputs of the same step
    (`accuracy`).  The oracle is the checker here, never the thing measured."""
    O = _oracle()
    t0 = time.perf_counter()
    ref = []
    for s in sets:
        ref.append((O.nufft_type1([s["x"], s["y"]], s["c"], N_MODES, eps=EPS),
                    O.nufft_type2([s["x"], s["y"]], s["f"], eps=EPS)))
    dt = time.perf_counter() - t0
    base = {"value": points_per_step(sets) / dt, "unit": "NU points/s", "cores": 1, "kind": "port",
            "sample": f"one full step (radial M={sets[0]['M']}, clustered M={sets[1]['M']}: one type 1 + one "
                      f"type 2 each), {dt:.1f} s"}
    rng = np.random.default_rng(2024)
    acc = {"eps": EPS, "dtype": "c64",
           "bound_vs_oracle": 2 * EPS,
           "bound_vs_direct": 10 * EPS + 2 * max(N_MODES) * 2.0 ** -24,
           "bound_note": "direct-sum bound = 10 eps + 2 N 2^-24: coordinates are folded in float32, as "
                         "nufftax does for complex64 inputs",
           "direct_sample": "type 1: 256 modes (16 x 16 product set, all points); type 2: 256 random "
                            "targets (all modes)"}
    for s, (f1, c2), (r1, r2) in zip(sets, gpu_out, ref):
        ax = [np.sort(rng.choice(np.arange(-(n // 2), (n - 1) // 2 + 1), 16, replace=False)) for n in N_MODES]
        d1 = O.direct_type1_product([s["x"], s["y"]], s["c"], ax, isign=1)
        sub1 = f1[np.ix_(ax[1] + N_MODES[1] // 2, ax[0] + N_MODES[0] // 2)]
        rows = np.sort(rng.choice(s["M"], 256, replace=False))
        d2 = O.direct_type2_points([s["x"][rows], s["y"][rows]], s["f"], isign=-1)
        acc[s["name"]] = {"type1_vs_oracle": O.rel_l2(f1, r1), "type2_vs_oracle": O.rel_l2(c2, r2),
                          "type1_vs_direct": O.rel_l2(sub1, d1), "type2_vs_direct": O.rel_l2(c2[rows], d2),
                          "oracle_type1_vs_direct": O.rel_l2(r1[np.ix_(ax[1] + N_MODES[1] // 2,
                                                                      ax[0] + N_MODES[0] // 2)], d1),
                          "oracle_type2_vs_direct": O.rel_l2(r2[rows], d2)}
    return base, acc


def _spread_chunk(args):
    O = _oracle()
    x, y, c, nf, kp = args
    return O.spread([O.premod(x), O.premod(y)], c, nf, kp)


def _interp_chunk(args):
    O = _oracle()
    x, y, fw, kp = args
    return O.interp([O.premod(x), O.premod(y)], fw, kp)


def run_reference(args):
    """Time the CPU restatement with every host core (process pool over point chunks)."""
    import multiprocessing as mp

    import scipy.fft as sfft

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O = _oracle()
    cores = os.cpu_count() or 1
    sets = workload(seed=1234)
    sample = []
    for s in sets:
        m = 131072 if s["name"] == "radial" else 524288
        sample.append({**s, "x": s["x"][:m], "y": s["y"][:m], "c": s["c"][:m], "M": m})
    kp = O.compute_kernel_params(EPS)
    nf = [O.compute_grid_size(n, 2.0, kp.nspread) for n in N_MODES]
    ph = [O.kernel_fourier_series(n, kp.nspread, kp.beta, kp.c) for n in nf]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        def one_step():
            for s in sample:
                ch = np.array_split(np.arange(s["M"]), cores)
                parts = pool.map(_spread_chunk, [(s["x"][i], s["y"][i], s["c"][i], nf, kp) for i in ch])
                fw = np.sum(parts, axis=0)
                O.deconvolve_shuffle(sfft.ifftn(fw, workers=cores) * (nf[0] * nf[1]), ph, N_MODES)
                fwh = O.deconvolve_pad(s["f"], ph, nf)
                fw2 = sfft.fftn(fwh, workers=cores)
                pool.map(_interp_chunk, [(s["x"][i], s["y"][i], fw2, kp) for i in ch])

        for _ in range(args.warmup):
            one_step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            one_step()
        dt = time.perf_counter() - t0
    pts = points_per_step(sample) * args.steps
    value = pts / dt
    line = {
        "metric": METRIC, "value": value, "unit": "NU points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": DATA,
        "config": bench_config(world, sets),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "NU points/s", "cores": cores, "kind": "port",
                         "sample": f"each step: radial first {sample[0]['M']} + clustered first {sample[1]['M']} "
                                   "points of the workload, one type 1 + one type 2 each (points/s counts the "
                                   "sample's points)"},
        "e2e": {"value": value, "unit": "NU points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_case(args):
    """One point set (a 2D set of the bench, or 8M uniform 3D points on 128^3
    modes), `reps` rounds of sort + type 1 + type 2, no timing: for ncu captures."""
    import torch

    import nufftax_b200 as nb

    dev = torch.device("cuda", 0)
    if args.case == "uniform3d":
        # 3D: M = 8e6 uniform points, 128^3 modes (nf 256^3), eps 1e-6, complex64
        M, N3 = int(8_000_000 * args.scale), (128, 128, 128)
        rng = np.random.default_rng(4)
        X = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev) for _ in range(3)]
        c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
        f = torch.from_numpy((rng.standard_normal(N3) + 1j * rng.standard_normal(N3)).astype(np.complex64)).to(dev)

        def one():
            nb.sort_cache.clear()
            nb.nufft3d1(*X, c, N3, eps=EPS)
            nb.nufft3d2(*X, f, eps=EPS)
    else:
        s = [s for s in workload(seed=1234, scale=args.scale) if s["name"] == args.case][0]
        M = s["M"]
        x, y = torch.from_numpy(s["x"]).to(dev), torch.from_numpy(s["y"]).to(dev)
        c, f = torch.from_numpy(s["c"]).to(dev), torch.from_numpy(s["f"]).to(dev)

        def one():
            nb.sort_cache.clear()
            nb.nufft2d1(x, y, c, N_MODES, eps=EPS)
            nb.nufft2d2(x, y, f, eps=EPS)
    for _ in range(args.reps):
        one()
    torch.cuda.synchronize()
    out = {"case": args.case, "M": M, "reps": args.reps}
    if args.time_calls:
        # per-call device time on one stream (CUDA events around each library call)
        from nufftax_b200 import profiling

        with profiling.record() as rec:
            for _ in range(args.reps):
                one()
        torch.cuda.synchronize()
        out["us_per_call"] = {k: round(1e3 * v["ms"] / max(v["calls"], 1), 2) for k, v in rec.summary().items()}
    print(json.dumps(out))


def batched_workload(seed=77, P=64):
    """64 problems: M log-uniform in [1e4, 2e6], modes per axis from {128, 256, 384, 512},
    even problems uniform, odd problems clustered N(0, 0.3^2)."""
    rng = np.random.default_rng(seed)
    probs = []
    for p in range(P):
        M = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        if p % 2:
            x, y = clustered_points(M, rng)
        else:
            x, y = rng.uniform(-np.pi, np.pi, (2, M)).astype(np.float32)
        nm = (int(rng.choice([128, 256, 384, 512])), int(rng.choice([128, 256, 384, 512])))
        c = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
        f = (rng.standard_normal((nm[1], nm[0])) + 1j * rng.standard_normal((nm[1], nm[0]))).astype(np.complex64)
        probs.append({"x": x, "y": y, "c": c, "f": f, "M": M, "n_modes": nm})
    return probs


def measure_batched(dev, steps: int, warmup: int, autotune: bool = False) -> dict:
    """Batched plan (one persistent launch per pass, CUDA graph) vs the per-problem plain path."""
    import torch

    import nufftax_b200 as nb
    from nufftax_b200.autotune import tune
    from nufftax_b200.batch import BatchPlan

    eps = 1e-5
    probs = batched_workload()
    d = [{k: (torch.from_numpy(v).to(dev) if isinstance(v, np.ndarray) else v) for k, v in q.items()} for q in probs]
    pts = sum(2 * q["M"] for q in probs)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def plain_step():
        nb.sort_cache.clear()
        for q in d:
            nb.nufft2d1(q["x"], q["y"], q["c"], q["n_modes"], eps=eps)
            nb.nufft2d2(q["x"], q["y"], q["f"], eps=eps)

    def timed(fn):
        warm(fn, warmup, 0.5)  # under the clock sampler (the caller's clocked block)
        tot = 0.0
        for i in range(steps):
            flush.fill_(float(i))
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / steps

    kp = nb.compute_kernel_params(eps)

    def make_plan(tiles=None, maxsubs=None, imodes=None):
        plan = BatchPlan([[q["x"], q["y"]] for q in d], [q["n_modes"] for q in d], eps=eps, tiles=tiles,
                         max_subproblem=maxsubs, interp_modes=imodes, graph=True)
        for p, q in enumerate(d):
            plan.c_in[p].copy_(q["c"])
            plan.f_in[p].copy_(q["f"])
        return plan

    plan = make_plan()
    tuned = None
    if autotune:
        # tile, subproblem size and threads per point tuned per problem class
        tiles, maxsubs, imodes = [], [], []
        for q in d:
            nf = tuple(nb.compute_grid_size(n, 2.0, kp.nspread) for n in q["n_modes"])
            t, m, modes = tune([q["x"], q["y"]], nf, kp)
            tiles.append(t)
            maxsubs.append(m)
            imodes.append(modes[1])
        tuned = make_plan(tiles, maxsubs, imodes)
    with clocked(dev.index) as ck:
        plain_ms = timed(plain_step)
        batch_ms = timed(lambda: plan.run())
        tuned_ms = timed(lambda: tuned.run()) if tuned is not None else None
    best_ms = min(batch_ms, tuned_ms) if tuned_ms is not None else batch_ms
    out = {"metric": "batched 2D type-1 + type-2 NU points/s (64 problems, eps 1e-5, complex64)",
            "value": pts / (best_ms / 1e3), "unit": "NU points/s", "plain_value": pts / (plain_ms / 1e3),
            "speedup_vs_plain": plain_ms / best_ms, "ms_per_step": best_ms, "plain_ms_per_step": plain_ms,
            "default_tiling_ms_per_step": batch_ms, "points_per_step": pts, "steps": steps, "warmup": warmup,
            "autotune": bool(autotune), "clocks": ck.summary,
            "config": {"workload": "64 problems, M log-uniform [1e4, 2e6], modes per axis from {128,256,384,512}, "
                                   "half uniform / half clustered N(0,0.3^2), sort included every step",
                       "l2": "flushed between steps"}}
    if tuned_ms is not None:
        out["tuned_ms_per_step"] = tuned_ms
        out["tuned_wins"] = tuned_ms < batch_ms
    return out


def run_batched(args):
    import torch

    print(json.dumps(measure_batched(torch.device("cuda", 0), args.steps, args.warmup, args.autotune)), flush=True)


def measure_grad3d(dev, steps: int, warmup: int, M: int = 8_000_000) -> dict:
    """3D type 1, M uniform points, 128^3 modes, eps 1e-6, complex64:
    loss = ||nufft3d1(x, y, z, c) - f_target||^2 and its gradients w.r.t. c, x, y, z
    through the hand-written adjoint kernels (forward + backward per step).
    Inputs are drawn on the device (seeded)."""
    import torch

    import nufftax_b200 as nb

    N, eps = (128, 128, 128), 1e-6
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    X = [(torch.rand(M, device=dev, generator=g) * 2 - 1) * np.pi for _ in range(3)]
    c = torch.complex(torch.randn(M, device=dev, generator=g), torch.randn(M, device=dev, generator=g))
    tgt = torch.complex(torch.randn(N[::-1], device=dev, generator=g), torch.randn(N[::-1], device=dev, generator=g))

    def step():
        nb.sort_cache.clear()
        xs = [x.detach().requires_grad_(True) for x in X]
        cc = c.detach().requires_grad_(True)
        f = nb.nufft3d1(*xs, cc, N, eps=eps)
        loss = (f - tgt).abs().pow(2).sum()
        loss.backward()
        return loss, cc.grad, [x.grad for x in xs]

    tot = 0.0
    with clocked(dev.index) as ck:
        warmup = warm(step, warmup)
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            step()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
    ms = tot / steps
    return {"metric": "differentiated 3D type-1 NU points/s (forward + backward w.r.t. c, x, y, z)",
            "value": M / (ms / 1e3), "unit": "NU points/s", "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "clocks": ck.summary,
            "config": {"workload": f"M={M} uniform 3D, 128^3 modes, nf 256^3, eps 1e-6, complex64, "
                                   "loss ||f - t||^2, gradients w.r.t. c, x, y, z; sort every step"}}


def run_grad3d(args):
    import torch

    dev = torch.device("cuda", 0)
    M = int(8_000_000 * args.scale)
    line = measure_grad3d(dev, args.steps, args.warmup, M)
    if args.check:
        line["check"] = grad3d_check(M, (128, 128, 128), np.random.default_rng(4))
    print(json.dumps(line), flush=True)


def grad3d_check(M, N, rng):
    import torch

    import nufftax_b200 as nb

    dev = torch.device("cuda", 0)
    out = {}
    # (1) central finite differences, complex128, 32 random entries (both sides
    # differentiate the same approximate transform, so eps does not limit agreement)
    eps = 1e-7
    X = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).to(dev) for _ in range(3)]
    c = torch.from_numpy(rng.standard_normal(M) + 1j * rng.standard_normal(M)).to(dev)
    tgt = torch.from_numpy(rng.standard_normal(N[::-1]) + 1j * rng.standard_normal(N[::-1])).to(dev)
    xs = [x.clone().requires_grad_(True) for x in X]
    cc = c.clone().requires_grad_(True)
    loss = (nb.nufft3d1(*xs, cc, N, eps=eps) - tgt).abs().pow(2).sum()
    loss.backward()

    def L():
        with torch.no_grad():
            return float((nb.nufft3d1(*xs, cc, N, eps=eps) - tgt).abs().pow(2).sum())

    h = 1e-4
    errs = []
    for e in range(32):
        j = int(rng.integers(M))
        which = e % 5  # c.re, c.im, x, y, z
        with torch.no_grad():
            if which < 2:
                unit = 1.0 if which == 0 else 1j
                base = cc[j].item()
                cc[j] = base + unit * h
                lp = L()
                cc[j] = base - unit * h
                lm = L()
                cc[j] = base
                an = cc.grad[j].real.item() if which == 0 else cc.grad[j].imag.item()
            else:
                t = xs[which - 2]
                base = t[j].item()
                t[j] = base + h
                lp = L()
                t[j] = base - h
                lm = L()
                t[j] = base
                an = t.grad[j].item()
        fd = (lp - lm) / (2 * h)
        errs.append(abs(an - fd) / max(abs(fd), 1e-300))
    out["fd_c128_h1e-4_max_rel_err"] = max(errs)
    out["fd_c128_h1e-4_median_rel_err"] = float(np.median(errs))
    # (2) spectral formula of the reference (complex64 forward, eps 1e-6)
    x32 = [x.float().requires_grad_(True) for x in X]
    c64 = c.to(torch.complex64).requires_grad_(True)
    t64 = tgt.to(torch.complex64)
    f = nb.nufft3d1(*x32, c64, N, eps=1e-6)
    G = 2 * (f.detach() - t64)
    (f - t64).abs().pow(2).sum().backward()
    rel = []
    for d in range(3):
        k = torch.arange(-(N[d] // 2), (N[d] - 1) // 2 + 1, device=dev, dtype=torch.float32)
        shape = [1, 1, 1]
        shape[2 - d] = N[d]
        t2 = nb.nufft3d2(*[x.detach() for x in x32], (-1j * k.reshape(shape)) * G, eps=1e-6, isign=-1)
        ref = (c64.detach().conj() * t2).real
        rel.append(float((x32[d].grad - ref).norm() / ref.norm()))
    dc_ref = nb.nufft3d2(*[x.detach() for x in x32], G, eps=1e-6, isign=-1)
    out["spectral_formula_rel_l2_dx_dy_dz"] = rel
    out["spectral_formula_rel_l2_dc"] = float((c64.grad - dc_ref).norm() / dc_ref.norm())
    return out


class _DevicePool:
    """Pre-drawn device random numbers that the served requests' inputs are
    sliced from (no kernel launches per request, the same cost in the served
    and the one-at-a-time paths): uniform coordinates in [-pi, pi), target
    frequencies in [-300, 300) and standard normals viewed as complex."""

    _pools: dict = {}

    def __init__(self, device, n_uniform=1 << 26, n_normal=1 << 27):
        import torch

        g = torch.Generator(device=device)
        g.manual_seed(5)
        self.u = (torch.rand(n_uniform, device=device, generator=g) * 2 - 1) * np.pi
        self.t = self.u * (300.0 / np.pi)
        self.n = torch.randn(n_normal, device=device, generator=g)

    @classmethod
    def get(cls, device):
        key = str(device)
        if key not in cls._pools:
            cls._pools[key] = cls(device)
        return cls._pools[key]


def served_requests(n, seed=5):
    """The served mix: 50 % 2D type 1/2 (modes per axis from 128..512 in steps of
    32, M log-uniform 1e3..4e6), 30 % 3D type 1/2 (modes per axis from 64..160 in
    steps of 16, M log-uniform 1e4..8e6),
    20 % 2D type 3 (sources uniform in [-pi, pi)^2, targets uniform in
    [-300, 300]^2, M = K log-uniform 1e3..1e6); eps 1e-6, complex64.  Inputs are
    slices, at seeded offsets, of random numbers drawn on the device once."""
    import torch

    from nufftax_b200 import compute_type3_grid_sizes_2d
    from nufftax_b200.serve import Request

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        u = rng.random()
        kind = int(rng.integers(1, 3))
        if u < 0.5:
            dim = 2
            M = int(np.exp(rng.uniform(np.log(1e3), np.log(4e6))))
            nm = tuple(int(rng.choice(np.arange(128, 513, 32))) for _ in range(2))
        elif u < 0.8:
            dim = 3
            M = int(np.exp(rng.uniform(np.log(1e4), np.log(8e6))))
            nm = tuple(int(rng.choice(np.arange(64, 161, 16))) for _ in range(3))
        else:
            dim, kind = 2, 3
            M = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
            nm = compute_type3_grid_sizes_2d(np.pi, np.pi, 300.0, 300.0, eps=1e-6)

        def make(device, kind=kind, dim=dim, M=M, nm=nm, sd=int(rng.integers(1 << 31))):
            pool = _DevicePool.get(device)
            r = np.random.default_rng(sd)
            off = lambda n_, total: 2 * int(r.integers(0, (total - n_) // 2))  # noqa: E731 (even: complex views)
            X = [pool.u[o:o + M] for o in (off(M, pool.u.numel()) for _ in range(dim))]
            if kind == 2:
                shape = tuple(reversed(nm))
                k = math.prod(shape)
                o = off(2 * k, pool.n.numel())
                return X, torch.view_as_complex(pool.n[o:o + 2 * k].view(k, 2)).view(shape), None
            o = off(2 * M, pool.n.numel())
            c = torch.view_as_complex(pool.n[o:o + 2 * M].view(M, 2))
            T = [pool.t[o2:o2 + M] for o2 in (off(M, pool.t.numel()) for _ in range(dim))] if kind == 3 else None
            return X, c, T

        reqs.append(Request(kind=kind, dim=dim, n_modes=nm, M=M, K=M if kind == 3 else 0, make_inputs=make))
    return reqs


def measure_serve(dev, n: int, plain_sample: int, loads, slots: int = 8) -> dict:
    """Served stream vs one-at-a-time plain execution; Poisson arrivals."""
    import copy

    import torch

    import nufftax_b200 as nb
    from nufftax_b200.serve import NufftServer

    reqs = served_requests(n)
    # both paths start with warm cuFFT plans: one small transform per distinct shape
    shapes = sorted({(r.kind, r.dim, tuple(r.n_modes)) for r in reqs})
    for kind, dim, nm in shapes:
        g = torch.Generator(device=dev)
        X = [torch.rand(64, device=dev, generator=g) for _ in range(dim)]
        if kind == 3:
            c = torch.ones(64, dtype=torch.complex64, device=dev)
            nb.nufft2d3(*X, c, *[x * 300 for x in X], nm)
        elif kind == 1:
            {2: nb.nufft2d1, 3: nb.nufft3d1}[dim](*X, torch.ones(64, dtype=torch.complex64, device=dev), nm)
        else:
            {2: nb.nufft2d2, 3: nb.nufft3d2}[dim](*X, torch.ones(tuple(reversed(nm)), dtype=torch.complex64,
                                                                device=dev))
    torch.cuda.synchronize()
    # one-at-a-time: each request alone through the public API, synchronised
    sample = [copy.copy(r) for r in reqs[: min(n, plain_sample)]]
    for r in sample[:5]:
        _plain(nb, r, dev)
    torch.cuda.synchronize()
    with clocked(dev.index) as ck:
        t0 = time.perf_counter()
        for r in sample:
            _plain(nb, r, dev)
            torch.cuda.synchronize()
        plain_s = time.perf_counter() - t0
        plain_pts = sum(r.points() for r in sample) / plain_s
        plain_rps = len(sample) / plain_s
        out = {"metric": "served mixed stream NU points/s (p50/p99 latency)", "unit": "NU points/s",
               "requests": n, "distinct_shapes": len(shapes),
               "one_at_a_time": {"points_per_s": plain_pts, "requests_per_s": plain_rps, "sample": len(sample)},
               "loads": []}
        rng = np.random.default_rng(11)
        for load in loads:
            rate = load * plain_rps
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
            server = NufftServer(dev, slots=slots, hbm_budget=150e9, keep_results=False)
            batch = [copy.copy(r) for r in reqs]
            # warm the caches (plans, grid pool) with the first few requests
            server.serve([copy.copy(r) for r in reqs[:20]])
            torch.cuda.synchronize()
            server.completed = []
            retries0 = torch.cuda.memory_stats(dev).get("num_alloc_retries", 0)
            torch.cuda.reset_peak_memory_stats(dev)
            done = server.serve(batch, list(arrivals))
            st = server.stats(done)
            mem = torch.cuda.memory_stats(dev)
            # allocator retries free the cache and synchronise the device: a stall
            st["alloc_retries"] = int(mem.get("num_alloc_retries", 0) - retries0)
            st["peak_reserved_gb"] = round(mem.get("reserved_bytes.all.peak", 0) / 1e9, 1)
            st["offered_load"] = load
            st["offered_requests_per_s"] = rate
            out["loads"].append(st)
    best = max(out["loads"], key=lambda d: d["points_per_s"])
    out["value"] = best["points_per_s"]
    out["p50_ms"] = best["p50_ms"]
    out["p99_ms"] = best["p99_ms"]
    out["speedup_vs_one_at_a_time"] = best["points_per_s"] / plain_pts
    out["clocks"] = ck.summary
    out["config"] = {"workload": "Poisson arrivals: 50% 2D type 1/2 (modes 128..512 per axis, M log-uniform 1e3..4e6), "
                                 "30% 3D type 1/2 (modes 64..160, M log-uniform 1e4..8e6), 20% 2D type 3 (targets in "
                                 "[-300,300]^2, M = K log-uniform 1e3..1e6), eps 1e-6, complex64, HBM budget 150 GB",
                     "offered_load": "multiples of the measured one-at-a-time request rate",
                     "inputs": "sliced at admission from random numbers drawn on the device once (seeded offsets), "
                               "the same in both paths"}
    return out


def run_serve(args):
    import torch

    print(json.dumps(measure_serve(torch.device("cuda", 0), args.requests, args.plain_sample, args.loads,
                                   args.slots)), flush=True)


def measure_1d(dev, steps: int, warmup: int) -> dict:
    """The 1D configuration: type 1 then type 2, M = 200,000 uniform points,
    N = 8192 modes, eps 1e-6, complex64 (sort included every step)."""
    import torch

    import nufftax_b200 as nb

    rng = np.random.default_rng(21)
    M, N = 200_000, 8192
    x = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
    f = torch.from_numpy((rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)).to(dev)

    def step():
        nb.sort_cache.clear()
        nb.nufft1d1(x, c, N, eps=EPS)
        nb.nufft1d2(x, f, eps=EPS)

    with clocked(dev.index) as ck:
        n_warm = warm(step, warmup)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            step()
        b.record()
        torch.cuda.synchronize()
        eager_ms = a.elapsed_time(b) / steps
        # the same step captured once through the public API and replayed
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            step()
        for _ in range(max(3, warmup)):
            graph.replay()
        torch.cuda.synchronize()
        a.record()
        for _ in range(steps):
            graph.replay()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        del graph
    return {"metric": "1D type-1 + type-2 NU points/s (M=200000, N=8192, eps 1e-6, complex64)", "value": 2 * M / (ms / 1e3),
            "unit": "NU points/s", "ms_per_step": ms, "steps": steps, "warmup": n_warm, "clocks": ck.summary,
            "eager_value": 2 * M / (eager_ms / 1e3), "eager_ms_per_step": eager_ms,
            "note": "inputs resident, back-to-back steps; value: the step replayed from a CUDA graph captured "
                    "through the public API (sort included); eager: launched from Python, launch-bound at this "
                    "size; warm-up runs 1 s under the clock sampler"}


def _plain(nb, r, dev):
    X, s, T = r.make_inputs(dev)
    if r.kind == 1:
        fn = {2: nb.nufft2d1, 3: nb.nufft3d1}[r.dim]
        return fn(*X, s, r.n_modes, eps=r.eps)
    if r.kind == 2:
        fn = {2: nb.nufft2d2, 3: nb.nufft3d2}[r.dim]
        return fn(*X, s, eps=r.eps)
    return nb.nufft2d3(*X, s, *T, r.n_modes, eps=r.eps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nufftax_b200", choices=["nufftax_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-subconfigs", action="store_true", help="headline only (no batched / grad3d / served / 1D)")
    ap.add_argument("--served-requests", type=int, default=1000, help="requests of the served sub-record")
    ap.add_argument("--case", choices=["radial", "clustered", "uniform3d"],
                    help="profile one point set only (no timing)")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--time-calls", action="store_true", help="with --case: also print per-call device time")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--config", choices=["default", "batched", "grad3d", "serve"], default="default")
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--plain-sample", type=int, default=1000)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--loads", type=float, nargs="+", default=[1.0, 2.0])
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--check", action="store_true")
    args = ap.parse_args()
    if args.config == "batched":
        run_batched(args)
        return
    if args.config == "grad3d":
        run_grad3d(args)
        return
    if args.config == "serve":
        run_serve(args)
        return
    if args.case:
        run_case(args)
        return
    if args.warmup < 3 and args.impl != "reference":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
