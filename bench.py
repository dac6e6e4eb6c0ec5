#!/usr/bin/env python3
"""Benchmark: AV1 post-filter chain (deblock -> CDEF -> loop restoration) on B200.

Workload (the post-filter stage micro-benchmark configuration): a batch of 64
frames of 1920x1080 8-bit 4:2:0 synthetic decoder state per GPU — planes from a
bilinearly upsampled 16x16 uniform field plus uniform noise in [-12, 12],
legal per-4x4 transform sizes, deblock levels 0..63 with sharpness 0..7,
per-64x64 CDEF strengths (cdef_bits 3, damping 3..6) and 64x64 restoration
units split Wiener / self-guided.  One step = the whole chain over the batch,
one launch per stage across the 64 frames.  `--bit-depth 10` runs the 10-bit
variant.

Printed JSON (rank 0): `value` is whole-job frames/s with inputs resident in
HBM; `e2e` is the same metric through the C-ABI with the inputs copied from
pinned host memory and the restored frames copied back every step; `roofline`
is the dominant kernel's algorithmic bytes per launch over its CUDA-event
duration against the measured HBM copy bandwidth; `cpu_baseline` is the CPU
oracle (a C restatement of the reference's CPU path) on a bounded sample.

`--impl reference` times the reference's CPU implementation of the path (the
same C restatement — the Rust crate does not build here) on all host cores.

Further sections in the same line (rank 0, one GPU): `recon_stages` (inter
residuals, inter prediction, the intra wavefront at 1080p and at 3840x2160
tiled), `extra_stages` (superres, film grain), `motion_field`, `decode` (the
reference's conformance streams through the stream decoder, digests checked),
`batching` (256 mixed streams through the serving engine, batched against the
per-frame path at equal lanes) and `serving` (Poisson arrivals of 30-300
frame streams at three loads, for the batching mix and for 3840x2160 10-bit).
`--section NAME` runs one of them alone (`recon`, `extra`, `motion_field`,
`decode`, `batching`, `serving`, and also `chain`: the chain alone at the
default launch shapes, and `e2e`: the end-to-end leg alone); `--no-serving`
skips the last two of the line.
"""
import argparse
import concurrent.futures as cf
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "oxideav-av1_b200"


def load_package():
    if "oxideav_av1_b200" in sys.modules:
        return sys.modules["oxideav_av1_b200"]
    spec = importlib.util.spec_from_file_location("oxideav_av1_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["oxideav_av1_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
sys.path.insert(0, str(ROOT))

from oxideav_av1_b200 import abi, synth  # noqa: E402

WIDTH, HEIGHT = 1920, 1080
# What the main line times: frames through the post-filter chain (deblock,
# CDEF, loop restoration) of already reconstructed planes, bit-exact with the
# oracle; whole-stream decoding is timed in the `decode` and `serving` sections.
METRIC = "post-filter chain frames/s (deblock+CDEF+LR, bit-exact)"
UNIT = "frames/s"


def frame_seed(rank, i):
    return 1_000_003 * (rank + 1) + i


def max_over_ranks(ms, world, device):
    """The slowest rank's time: each rank's own device-timed milliseconds,
    all-reduced with MAX over the process group (one process per GPU)."""
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, frames_per_rank, ms_per_step):
    """Whole-job frames/s: every rank's frames over the slowest rank's step."""
    return world * frames_per_rank / (ms_per_step / 1e3)


def make_frames(rank, n, bit_depth):
    return [synth.make_frame(frame_seed(rank, i), WIDTH, HEIGHT, bit_depth=bit_depth) for i in range(n)]


def algorithmic_bytes(frame):
    """Per-frame algorithmic bytes of each stage (the path's roofline model).

    S bytes/sample, P samples of the cropped frame, M mi cells, U LR units:
      deblock  2*P*S + 10*M      (planes read+write; ~10 B of mi side data per 4x4)
      cdef     2*P*S + M + 64*SB (planes read+write; skip flags; one index per 64x64)
      lr       2*P*S + P*S/16 + 10*U (CDEF frame read, output write, 2+2 deblocked rows
                                    per 64-row stripe, unit parameters)
    """
    h = frame.hdr
    S = 2 if h.bit_depth > 8 else 1
    P = sum(frame.out_dims(p)[0] * frame.out_dims(p)[1] for p in range(h.num_planes))
    M = h.mi_rows * h.mi_cols
    SB = ((h.mi_rows + 15) // 16) * ((h.mi_cols + 15) // 16)
    U = sum(frame.lr_grid(p)[0] * frame.lr_grid(p)[1] for p in range(h.num_planes))
    return {"deblock": 2 * P * S + 10 * M, "cdef": 2 * P * S + M + 64 * SB, "lr": 2 * P * S + P * S // 16 + 10 * U}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic(kernel, workload, kind=None):
    """Per-frame DRAM bytes (kind None) or warp instructions (kind "inst") of
    `kernel` from the committed ncu summary, or None."""
    p = ROOT / "profiles" / "dram_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if line.startswith("#"):
            continue
        if kind:
            if len(parts) >= 4 and parts[0] == kind and parts[1] == kernel and parts[2] == workload:
                return int(parts[3])
        elif len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            return int(parts[2])
    return None


SMS, SCHEDULERS_PER_SM = 148, 4


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        self.first = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        # return once the tool has started and printed a sample (at most 5 s):
        # its start-up talks to the driver, which must not overlap timed work
        import select
        if select.select([self.proc.stdout], [], [], 5.0)[0]:
            line = self.proc.stdout.readline()
            if line.strip():
                self.first.append(line)
        return self

    def __exit__(self, *exc):
        self.lines = list(getattr(self, "first", []))
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines += [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# reference arm and CPU baseline: the C oracle on host cores
# ----------------------------------------------------------------------------

def cpu_time_frames(frames, threads):
    import oracle
    oracle.load()
    t0 = time.perf_counter()
    if threads == 1:
        for f in frames:
            oracle.postfilter_frame(f)
    else:
        with cf.ThreadPoolExecutor(threads) as ex:  # ctypes releases the GIL during the C call
            list(ex.map(oracle.postfilter_frame, frames))
    return time.perf_counter() - t0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # the GPU arm's batch: the same seeds, all of it every step
    frames = make_frames(0, args.frames, args.bit_depth)
    for _ in range(args.warmup):
        cpu_time_frames(frames, threads)
    dt = 0.0
    for _ in range(args.steps):
        dt += cpu_time_frames(frames, threads)
    value = len(frames) * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8" if args.bit_depth == 8 else "u16",
        "data": "synthetic",
        "config": config_block(args, frames_per_step=len(frames)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the whole {len(frames)}-frame workload per step on {threads} threads "
                                   "(one frame per task), full deblock+CDEF+LR chain (C restatement of the "
                                   "reference CPU path)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_block(args, frames_per_step):
    return {"workload": f"post-filter chain (deblock+CDEF+loop restoration), {frames_per_step} x "
                        f"{WIDTH}x{HEIGHT} {args.bit_depth}-bit 4:2:0 frames per GPU per step",
            "frames_per_step_per_gpu": frames_per_step, "resolution": f"{WIDTH}x{HEIGHT}",
            "bit_depth": args.bit_depth, "chroma": "4:2:0", "stages": ["deblock", "cdef", "lr"],
            "launch": "one launch per stage across the batch",
            "parallelism": f"independent frame batches per GPU (replicas, no collective), {args.gpus} GPU(s)",
            "l2": "inputs larger than L2 (each step reads ~200 MB of planes per GPU)"}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------

def run_gpu(args):
    import torch
    import torch.distributed as dist
    from oxideav_av1_b200 import postfilter

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    abi.load()
    frames = make_frames(rank, args.frames, args.bit_depth)
    dframes = [postfilter.DeviceFrame(f, device=dev) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    lib = abi.load()
    stream = torch.cuda.Stream(device=dev)
    sp = C.c_void_p(stream.cuda_stream)
    n = len(dframes)
    stages = [("deblock", lib.av1g_run_deblock), ("cdef", lib.av1g_run_cdef), ("lr", lib.av1g_run_lr)]

    # launch shapes: the project's autotuner times every candidate grid size
    # (and superres tile width) on this batch before the warm-up
    autotune = run_autotune(lib, jobs, n, stream, args.bit_depth > 8)

    def step(events=None):
        for i, (_, fn) in enumerate(stages):
            abi.check(fn(jobs, n, sp))
            if events is not None:
                events[i].record(stream)

    # clocks sampled over the warm-up, the timed steps and the per-frame / e2e
    # runs that follow; started (and settled) before the warm-up
    clk = ClockSampler(local)
    clk.__enter__()
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_stage = [[torch.cuda.Event(enable_timing=True) for _ in stages] for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        # a ~100 ms spin ahead of the first event keeps the stream busy while
        # the host enqueues the steps, so a host pause there cannot open an
        # idle gap inside the timed region (the spin itself is not timed; a
        # 20 ms spin was once outlasted by a ~45 ms host stall)
        torch.cuda._sleep(200_000_000)
        for k in range(args.steps):
            ev_start[k].record(stream)
            step(ev_stage[k])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    stage_ms = {name: 0.0 for name, _ in stages}
    total_ms = 0.0
    for k in range(args.steps):
        prev = ev_start[k]
        for i, (name, _) in enumerate(stages):
            d = prev.elapsed_time(ev_stage[k][i])
            stage_ms[name] += d
            total_ms += d
            prev = ev_stage[k][i]
    total_ms = max_over_ranks(total_ms, world, dev)
    ms_per_step = total_ms / args.steps
    value = job_rate(world, n, ms_per_step)

    # plain one-frame-per-launch path (same kernels, a launch per stage per frame)
    with torch.cuda.stream(stream):
        postfilter.run_postfilter(dframes, mode=abi.MODE_PER_FRAME, stream=stream, jobs=jobs)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            postfilter.run_postfilter(dframes, mode=abi.MODE_PER_FRAME, stream=stream, jobs=jobs)
        e1.record(stream)
    torch.cuda.synchronize()
    per_frame_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    graph = run_graphs(lib, jobs, n, stream, args.steps, world, dev)
    # end to end through av1g_run_postfilter (frame records prepared and
    # uploaded every call, as for new frames), and the same copies around
    # replays of a captured chain per group of frames
    e2e = run_e2e(args, frames, dframes, jobs, stream, dev, world, graphs=False)
    e2e["graph_variant"] = run_e2e(args, frames, dframes, jobs, stream, dev, world, graphs=True)
    clk.__exit__(None, None, None)
    clocks = clk.summary()

    # roofline of the dominant kernel
    ab = algorithmic_bytes(frames[0])
    dom = max(stage_ms, key=stage_ms.get)
    launch_ms = stage_ms[dom] / args.steps
    achieved = ab[dom] * n / (launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    kernel_name = {"deblock": "deblock_kernel", "cdef": "cdef_kernel", "lr": "lr_kernel"}[dom]
    workload = f"{WIDTH}x{HEIGHT}x{args.bit_depth}b"
    traffic = dram_traffic(kernel_name, workload)
    if traffic is not None:
        traffic = traffic * n  # summary holds bytes per frame
    inst = dram_traffic(kernel_name, workload, "inst")
    issue = None
    if inst is not None and clocks.get("sm_mhz"):
        peak_inst = SMS * SCHEDULERS_PER_SM * clocks["sm_mhz"] * 1e6
        ach_inst = inst * n / (launch_ms / 1e3)
        issue = {"achieved_warp_inst_per_s": ach_inst, "peak_warp_inst_per_s": peak_inst,
                 "frac": ach_inst / peak_inst,
                 "note": "the kernel's real ceiling: 148 SMs x 4 warp instructions per clock at the sampled SM "
                         "clock; instruction count from the committed ncu capture"}
    stage_frac = {}
    for name in stage_ms:
        a = ab[name] * n / (stage_ms[name] / args.steps / 1e3) / 1e9
        stage_frac[name] = {"ms_per_launch": stage_ms[name] / args.steps, "achieved_gbs": a, "frac": a / peak}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8" if args.bit_depth == 8 else "u16", "data": "synthetic",
        "config": config_block(args, n),
        "roofline": {"bound": "hbm", "kernel": kernel_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6650 GB/s", "issue": issue},
        "stages": stage_frac,
        "per_frame_path": {"value": job_rate(world, n, per_frame_ms), "unit": UNIT, "ms_per_step": per_frame_ms,
                           "launches_per_step": None},
        "graph": graph,
        "autotune": autotune,
        "e2e": e2e,
        # deblock is two kernels (edge-code prep + filter), CDEF and LR one each
        "gpu_launches": (len(stages) + 1) * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        line["recon_stages"] = run_recon_stages(args, dev, stream)
        line["extra_stages"] = run_extra_stages(args, dev, stream)
        line["motion_field"] = run_motion_field(args, dev, stream)
    if rank == 0 and world == 1:
        line["decode"] = run_decode(args, local)
    if rank == 0 and world == 1 and not args.no_serving:
        mix = mix_templates()
        line["batching"] = run_batching(args, local, mix)
        line["serving"] = run_serving(args, local, mix)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        k = args.cpu_sample
        dt = cpu_time_frames(frames[:k], 1)
        line["cpu_baseline"] = {"value": k / dt, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{k} of the {n} workload frames through the full chain, one thread"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_autotune(lib, jobs, n, stream, hbd):
    """av1g_autotune_postfilter on the batch; returns the chosen shape per stage."""
    t0 = time.perf_counter()
    abi.check(lib.av1g_autotune_postfilter(jobs, n, C.c_void_p(stream.cuda_stream), None))
    out = {"seconds": time.perf_counter() - t0}
    for st, name in enumerate(["deblock", "cdef", "superres", "lr", "film_grain"]):
        c, t = C.c_int32(), C.c_int32()
        abi.check(lib.av1g_autotune_get(st, int(hbd), C.byref(c), C.byref(t)))
        out[name] = {"ctas_per_sm": c.value} | ({"tile": t.value} if st == 2 else {})
    return out


def run_graphs(lib, jobs, n, stream, steps, world=1, dev=None):
    """The same chain (deblock, CDEF, LR) captured once as a CUDA graph
    (av1g_chain_graph_create) and replayed: batched (one launch per stage)
    and per-frame (a launch per stage per frame, all inside the graph)."""
    import torch
    sp = C.c_void_p(stream.cuda_stream)
    mask = (1 << 0) | (1 << 1) | (1 << 3)
    out = {}
    for name, mode in [("batched", abi.MODE_BATCHED), ("per_frame", abi.MODE_PER_FRAME)]:
        g = C.c_void_p()
        abi.check(lib.av1g_chain_graph_create(jobs, n, mask, mode, sp, C.byref(g)))
        try:
            for _ in range(3):
                abi.check(lib.av1g_chain_graph_launch(g, sp))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                for _ in range(steps):
                    abi.check(lib.av1g_chain_graph_launch(g, sp))
                e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
            out[name] = {"value": job_rate(world, n, ms), "unit": UNIT, "ms_per_step": ms,
                         "kernels_per_replay": lib.av1g_chain_graph_launches(g)}
        finally:
            abi.check(lib.av1g_chain_graph_destroy(g))
    return out


def _device_ms(stream, fn, reps=5):
    """Device time of the kernels fn() enqueues, and the host time of the call.

    A spin kernel holds the stream while the host prepares the launch (the
    library validates, plans and stages its records before it launches), so
    the events around the call bracket only the device work: the descriptor
    upload and the kernels."""
    import torch
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        fn()  # warm-up; also sizes the gate
    torch.cuda.synchronize()
    gate_ms = 3 * (time.perf_counter() - t0) * 1e3 + 5
    dev, host = [], []
    for _ in range(reps):
        with torch.cuda.stream(stream):
            torch.cuda._sleep(int(gate_ms * 2.0e6))  # ~gate_ms at up to 2 GHz
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h0 = time.perf_counter()
            fn()
            host.append((time.perf_counter() - h0) * 1e3)
            e1.record(stream)
        torch.cuda.synchronize()
        dev.append(e0.elapsed_time(e1))
    return min(dev), min(host)


def run_recon_stages(args, dev, stream):
    """Rows a1-a5 on one 1920x1080 frame each: the residual pass of inter
    blocks (dequant + inverse transform + merge), the inter prediction pass
    and the intra wavefront of a key frame (its residual pre-pass included).
    Device time per frame, the host time of the call beside it, and the
    algorithmic bytes over the device time."""
    from oxideav_av1_b200 import postfilter
    S = 2 if args.bit_depth > 8 else 1
    peak, _ = measured_peak()
    out = {}
    kw = dict(bit_depth=args.bit_depth)
    tw = np.array([4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64])
    th = np.array([4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16])

    rf = synth.make_recon_frame(9001, WIDTH, HEIGHT, **kw)
    d = postfilter.DeviceRecon(rf, device=dev)
    ms, hms = _device_ms(stream, lambda: postfilter.run_recon([d], stream=stream))
    area = int((tw[rf.tus["tx_size"]] * th[rf.tus["tx_size"]]).sum())
    nb = rf.coeffs.nbytes + len(rf.tus) * 16 + 2 * area * S
    out["residual"] = {"kernel": "recon_kernel", "ms_per_frame": ms, "host_ms_per_call": hms, "tus": len(rf.tus),
                       "algorithmic_bytes": nb, "achieved_gbs": nb / ms / 1e6, "frac_of_hbm": nb / ms / 1e6 / peak,
                       "bytes_model": "coefficients + TU records + the TU areas read and written"}

    ff = synth.make_inter_frame(9002, WIDTH, HEIGHT, **kw)
    d = postfilter.DeviceInter(ff, device=dev)
    ms, hms = _device_ms(stream, lambda: postfilter.run_inter([d], stream=stream))
    p = ff.preds
    nref = 1 + (p["kind"] == 1)
    nb = int(((p["w"].astype(np.int64) + 7) * (p["h"].astype(np.int64) + 7) * nref).sum() * S
             + (p["w"].astype(np.int64) * p["h"]).sum() * S)
    out["inter"] = {"kernel": "inter_kernel", "ms_per_frame": ms, "host_ms_per_call": hms, "calls": len(p),
                    "algorithmic_bytes": nb, "achieved_gbs": nb / ms / 1e6, "frac_of_hbm": nb / ms / 1e6 / peak,
                    "bytes_model": "sum over calls of (w+7)(h+7) per reference + w*h written"}

    fi = synth.make_intra_frame(9003, WIDTH, HEIGHT, **kw)
    d = postfilter.DeviceIntra(fi, device=dev)
    ms, _ = _device_ms(stream, lambda: postfilter.run_intra([d], stream=stream))
    # av1g_run_intra returns once its launch has finished (it reads the
    # per-frame wait status), so its host share is the call's wall time on an
    # idle stream less the device time
    import torch
    walls = []
    for _ in range(5):
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        postfilter.run_intra([d], stream=stream)
        walls.append((time.perf_counter() - h0) * 1e3)
    hms = max(0.0, min(walls) - ms)
    area = int((tw[fi.tus["tx_size"]] * th[fi.tus["tx_size"]]).sum())
    out["intra"] = {"kernels": ["intra_res_kernel", "intra_kernel"], "ms_per_frame": ms, "host_ms_per_call": hms,
                    "tus": len(fi.tus), "tus_per_us": len(fi.tus) / (ms * 1e3),
                    "bound": "latency: the TU dependency chain of the superblock wavefront",
                    "algorithmic_bytes": fi.coeffs.nbytes + 2 * area * S}
    # the full-reconstruction configuration's shape: 3840x2160 10-bit 4:2:0,
    # 128x128 superblocks — an inter frame's residual and prediction passes,
    # and a key frame with 2 x 2 tiles (the tiles' wavefronts run side by side)
    ru = synth.make_recon_frame(9011, 3840, 2160, bit_depth=10)
    du = postfilter.DeviceRecon(ru, device=dev)
    msu, hmsu = _device_ms(stream, lambda: postfilter.run_recon([du], stream=stream), reps=3)
    out["residual_uhd"] = {"kernel": "recon_kernel", "frame": "3840x2160 10-bit 4:2:0", "ms_per_frame": msu,
                           "host_ms_per_call": hmsu, "tus": len(ru.tus)}
    iu = synth.make_inter_frame(9012, 3840, 2160, bit_depth=10, sb_size=128)
    du = postfilter.DeviceInter(iu, device=dev)
    msu, hmsu = _device_ms(stream, lambda: postfilter.run_inter([du], stream=stream), reps=3)
    out["inter_uhd"] = {"kernel": "inter_kernel", "frame": "3840x2160 10-bit 4:2:0, 128x128 superblocks",
                        "ms_per_frame": msu, "host_ms_per_call": hmsu, "calls": len(iu.preds)}
    fu = synth.make_intra_frame(9004, 3840, 2160, bit_depth=10, sb_size=128, tiles=(1, 1))
    du = postfilter.DeviceIntra(fu, device=dev)
    msu, _ = _device_ms(stream, lambda: postfilter.run_intra([du], stream=stream), reps=3)
    out["intra_uhd"] = {"kernels": ["intra_res_kernel", "intra_kernel"], "frame": "3840x2160 10-bit 4:2:0, "
                        "128x128 superblocks, 2 x 2 tiles", "ms_per_frame": msu, "tus": len(fu.tus),
                        "tus_per_us": len(fu.tus) / (msu * 1e3)}
    return out


def run_extra_stages(args, dev, stream, templates=8, copies=6):
    """The post-filter stages the main batch leaves off: superres (2x
    horizontal upscale of the CDEF output and, with LR on, of the deblocked
    copy) and film grain (seeded parameters), each one launch over
    templates * copies 1920x1080 frames (more than L2 holds)."""
    import torch
    from oxideav_av1_b200 import postfilter
    S = 2 if args.bit_depth > 8 else 1
    peak, _ = measured_peak()
    lib = abi.load()
    sp = C.c_void_p(stream.cuda_stream)
    out = {}
    for name, kw, fn in [("superres", dict(superres_denom=16), lib.av1g_run_superres),
                         ("film_grain", dict(film_grain=True), lib.av1g_run_film_grain)]:
        tf = [synth.make_frame(9100 + k, WIDTH, HEIGHT, bit_depth=args.bit_depth, **kw) for k in range(templates)]
        frames = [tf[k % templates] for k in range(templates * copies)]
        dfr = [postfilter.DeviceFrame(f, device=dev) for f in frames]
        jobs = postfilter.jobs_array(dfr)
        n = len(dfr)
        shapes = run_autotune(lib, jobs, n, stream, args.bit_depth > 8)
        for _ in range(3):
            abi.check(fn(jobs, n, sp))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                abi.check(fn(jobs, n, sp))
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        h = frames[0].hdr
        P_up = sum(frames[0].out_dims(p)[0] * frames[0].out_dims(p)[1] for p in range(h.num_planes))
        if name == "superres":
            P_down = sum(frames[0].plane_dims(p)[0] * frames[0].plane_dims(p)[1] for p in range(h.num_planes))
            per = (P_down + P_up) * S * (2 if h.uses_lr else 1)
            model = "(downscaled + upscaled samples) per pass; two passes (CDEF output and deblocked copy) with LR on"
        else:
            per = 2 * P_up * S
            model = "output planes read and written once (grain templates and LUTs are per frame, negligible)"
        kern = "superres_kernel" if name == "superres" else "grain_template_kernel + grain_blend_kernel"
        out[name] = {"kernel": kern, "frames": n, "ms_per_launch": ms, "algorithmic_bytes_per_frame": per,
                     "launch_shape": shapes[name],
                     "achieved_gbs": per * n / ms / 1e6, "frac_of_hbm": per * n / ms / 1e6 / peak,
                     "bytes_model": model}
        del dfr, jobs
        torch.cuda.empty_cache()
    return out


def run_chain(args, dev, stream):
    """The post-filter chain alone (deblock, CDEF, loop restoration; one
    launch per stage over the batch), W untimed passes then K timed ones, at
    the default launch shapes: the command the per-kernel profiles capture."""
    from oxideav_av1_b200 import postfilter
    lib = abi.load()
    frames = make_frames(0, args.frames, args.bit_depth)
    dframes = [postfilter.DeviceFrame(f, device=dev) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    n = len(dframes)
    sp = C.c_void_p(stream.cuda_stream)
    stages = [lib.av1g_run_deblock, lib.av1g_run_cdef, lib.av1g_run_lr]
    import torch
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            for fn in stages:
                abi.check(fn(jobs, n, sp))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            for fn in stages:
                abi.check(fn(jobs, n, sp))
        e1.record(stream)
    torch.cuda.synchronize()
    return {"frames": n, "bit_depth": args.bit_depth, "ms_per_step": e0.elapsed_time(e1) / args.steps,
            "launches_per_step": 4}


def run_e2e_section(args, dev, stream):
    """The end-to-end leg alone, on the main line's frames and launch shapes:
    pinned-host inputs and outputs copied every step around the chain, through
    av1g_run_postfilter and through replays of captured chain graphs."""
    from oxideav_av1_b200 import postfilter
    lib = abi.load()
    frames = make_frames(0, args.frames, args.bit_depth)
    dframes = [postfilter.DeviceFrame(f, device=dev) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    run_autotune(lib, jobs, len(dframes), stream, args.bit_depth > 8)
    out = run_e2e(args, frames, dframes, jobs, stream, dev, 1, graphs=False)
    out["graph_variant"] = run_e2e(args, frames, dframes, jobs, stream, dev, 1, graphs=True)
    return out


def run_motion_field(args, dev, stream, frames=16):
    """Row f2 on 1920x1080 frames (mi 270 x 480): §7.19 storage of `frames`
    decoded frames in one launch, then the §7.9 projection of `frames`
    current frames (each from four stored slots, up to four passes) in one
    call.  Device time per frame beside the oracle's single-thread time per
    frame on the same inputs."""
    import torch
    from oxideav_av1_b200 import mfmv
    import oracle
    rows, cols = 270, 480
    cells, pos = rows * cols, (rows >> 1) * (cols >> 1)
    peak, _ = measured_peak()
    ins = [synth.make_mf_store_inputs(9200 + k, rows, cols) for k in range(frames)]
    store_jobs, store_keep = [], []
    for s in ins:
        rf, mv = torch.from_numpy(s["ref_frames"]).to(dev), torch.from_numpy(s["mvs"]).to(dev)
        j, r, m = mfmv.store_job(rows, cols, True, s["order_hint"], s["hint_bits"], s["ref_order_hint"], rf, mv)
        store_jobs.append(j)
        store_keep.append((rf, mv, r, m))
    ms_s, hms_s = _device_ms(stream, lambda: mfmv.run_store(store_jobs, stream=stream))
    scenes = [synth.make_mf_scene(9300 + k, rows, cols) for k in range(frames)]
    keep, pjobs = [], []
    for sc in scenes:
        slots = [None if sl is None else dict(sl, mf_mvs=torch.from_numpy(sl["mf_mvs"]).to(dev),
                                              mf_ref_frames=torch.from_numpy(sl["mf_ref_frames"]).to(dev))
                 for sl in sc["slots"]]
        j, out = mfmv.project_job(slots, sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"], sc["hint_bits"],
                                  rows, cols, device=dev)
        keep.append((slots, out))
        pjobs.append(j)
    ms_p, hms_p = _device_ms(stream, lambda: mfmv.run_project(pjobs, stream=stream))
    t0 = time.perf_counter()
    for s in ins[:4]:
        oracle.mf_store(rows, cols, True, s["order_hint"], s["hint_bits"], s["ref_order_hint"], s["ref_frames"],
                        s["mvs"])
    cpu_s = (time.perf_counter() - t0) * 1e3 / 4
    t0 = time.perf_counter()
    for sc in scenes[:4]:
        oracle.mf_project(sc["slots"], sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"], sc["hint_bits"],
                          rows, cols)
    cpu_p = (time.perf_counter() - t0) * 1e3 / 4
    nb_s = 15 * cells
    nb_p = 28 * pos + 8 * pos
    return {"frames_per_launch": frames,
            "store": {"kernel": "mf_store_kernel", "ms_per_frame": ms_s / frames, "host_ms_per_call": hms_s,
                      "algorithmic_bytes_per_frame": nb_s, "achieved_gbs": nb_s * frames / ms_s / 1e6,
                      "frac_of_hbm": nb_s * frames / ms_s / 1e6 / peak,
                      "cpu_baseline": {"kind": "port", "cores": 1, "ms_per_frame": cpu_s},
                      "bytes_model": "per 4x4 cell: RefFrames[2] + Mvs[2][2] read, MfRefFrames + MfMvs written"},
            "project": {"kernels": ["mf_claim_kernel", "mf_write_kernel"], "ms_per_frame": ms_p / frames,
                        "host_ms_per_call": hms_p, "algorithmic_bytes_per_frame": nb_p,
                        "achieved_gbs": nb_p * frames / ms_p / 1e6,
                        "frac_of_hbm": nb_p * frames / ms_p / 1e6 / peak,
                        "cpu_baseline": {"kind": "port", "cores": 1, "ms_per_frame": cpu_p},
                        "bytes_model": "per 8x8 position: 7 projected MVs written + one 8-byte claim word "
                                       "(stored candidates read per pass are L2-resident)"}}


# Whole-stream decoding through the serving engine's public API
# (av1g_stream_open / av1g_submit_frame / av1g_poll / av1g_fetch_output):
# host descriptors in, host frames out.

# The stream-batching configuration: 256 concurrent streams, resolutions
# 640x360 / 1280x720 / 1920x1080 / 3840x2160 weighted 4:3:2:1, 8- or 10-bit,
# 4:2:0 or 4:4:4, 8-60 frames each.
BATCH_SHAPES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]
BATCH_WEIGHTS = [4, 3, 2, 1]
# The serving configuration: 3840x2160 10-bit 4:2:0 streams of 30-300 frames,
# 25 % with film grain, Poisson arrivals (mean 40 streams/s), 120 GB budget.
SERVE_SHAPE = (3840, 2160, 10)
SERVE_RATE = 40.0
SERVE_BUDGET = 120 * 10**9
# a template is a key frame and inter frames; a longer stream cycles the
# inter frames (each references whatever the slots hold at that point, so
# the decode stays a valid, deterministic stream)
TEMPLATE_FRAMES = 3


def _make_template(spec):
    """One stream template; runs in a spawned worker process.  3840x2160
    streams use the full-reconstruction configuration's 2 x 2 tile grid."""
    seed, w, h, bd, ss, grain, sb = spec
    return synth.make_stream(seed, n_frames=TEMPLATE_FRAMES, width=w, height=h, bit_depth=bd, ssx=ss, ssy=ss,
                             film_grain=grain, sb_size=sb, tiles=(1, 1) if w >= 3840 else (0, 0))


def make_templates(specs):
    """Templates generated in parallel (synthesis is Python-bound) by spawned
    interpreters, which inherit no CUDA state; largest first."""
    import multiprocessing as mp
    order = sorted(range(len(specs)), key=lambda i: -specs[i][1] * specs[i][2] * (3 - specs[i][4]))
    with mp.get_context("spawn").Pool(max(1, min(len(specs), os.cpu_count() or 1))) as pool:
        res = pool.map(_make_template, [specs[i] for i in order], chunksize=1)
    out = [None] * len(specs)
    for i, r in zip(order, res):
        out[i] = r
    return out


def stream_frame(tpl, k):
    return tpl[0] if k == 0 else tpl[1 + (k - 1) % (len(tpl) - 1)]


def _fetch_digest(lib, h, ticket):
    """(status, digest of the frame's planes, latency ms); the digest (CRC-32
    and byte length of each plane: an equality check between two decodes of
    the same stream, at ~4 GB/s per client thread so that checking does not
    bound the measured rate) is taken on the engine's pinned output buffer,
    then the ticket is freed."""
    import zlib
    o = abi.FrameOut()
    st = lib.av1g_fetch_output(h, ticket, C.byref(o))
    dg = []
    if st == abi.AV1G_OK and o.shown:
        for p in range(o.num_planes):
            pl = o.planes[p]
            n = pl.stride * pl.height
            dg.append((zlib.crc32(memoryview((C.c_uint8 * n).from_address(pl.data))), n))
    lat = o.latency_ms
    lib.av1g_release_output(h, ticket)
    return st, tuple(dg), lat


def _fetch_only(lib, h, ticket):
    """(status, None, latency ms): the frame fetched (its planes are already
    in host memory) and freed, without checking its samples."""
    o = abi.FrameOut()
    st = lib.av1g_fetch_output(h, ticket, C.byref(o))
    lat = o.latency_ms
    lib.av1g_release_output(h, ticket)
    return st, None, lat


def drive(eng, templates, sbs, streams, clients=8, window=2, check=True):
    """Decodes `streams` [(template index, frame count)] through the engine.
    `clients` threads each own a group of streams, as a server's connections
    would: a client submits frame k of each of its streams in turn, keeps at
    most `window` frames per stream in flight (fetching the oldest first)
    and, when the engine answers AV1G_EBUSY, fetches before retrying.
    Returns (frames/s over the wall clock, per-stream frame digests,
    per-frame latencies in ms, every status OK)."""
    from collections import deque
    lib = eng.lib
    hs = [eng.open_stream(synth.stream_seq(templates[t], sbs[t])) for t, _ in streams]
    assert all(h is not None for h in hs), "budget too small for the stream set"
    groups = [list(range(g, len(streams), clients)) for g in range(min(clients, len(streams)))]
    failures = []  # (stream, frame, poll result, fetch status, error text)

    def client(group):
        inflight = deque()
        digests = {i: [] for i in group}
        lats, ok = [], True

        def fetch_oldest():
            nonlocal ok
            i, t = inflight.popleft()
            r = eng.poll(t, 300.0)
            st, dg, lat = (_fetch_digest if check else _fetch_only)(lib, hs[i].h, t)
            if r != abi.AV1G_OK or st != abi.AV1G_OK:
                ok = False
                failures.append((i, len(digests[i]), r, st, lib.av1g_last_error().decode(errors="replace")))
            digests[i].append(dg)
            lats.append(lat)

        for k in range(max(streams[i][1] for i in group)):
            for i in group:
                t, n = streams[i]
                if k >= n:
                    continue
                while len(inflight) >= window * len(group):
                    fetch_oldest()
                while True:
                    try:
                        inflight.append((i, hs[i].submit(stream_frame(templates[t], k))))
                        break
                    except abi.Av1gError as e:
                        if e.status != abi.AV1G_EBUSY:
                            raise
                        if inflight:
                            fetch_oldest()
                        else:
                            time.sleep(0.0005)
        while inflight:
            fetch_oldest()
        return digests, lats, ok

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(len(groups)) as ex:  # ctypes drops the GIL inside the engine calls
        results = list(ex.map(client, groups))
    dt = time.perf_counter() - t0
    for h in hs:
        h.close()
    digests, lats, ok = {}, [], True
    for d, l, o in results:
        digests.update(d)
        lats += l
        ok &= o
    if failures:
        sys.stderr.write(f"drive: {len(failures)} frames failed, first {failures[:4]}\n")
        FRAME_FAILURES.extend(failures)
    return sum(n for _, n in streams) / dt, [digests[i] for i in range(len(streams))], lats, ok


# Frames the engine failed during the current section (drive appends; the
# batching and serving sections report them in their results rather than
# stopping the run).
FRAME_FAILURES = []


def _failures_summary():
    return {"count": len(FRAME_FAILURES), "first": [list(f) for f in FRAME_FAILURES[:4]]}


def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * len(xs)))] if xs else None


def _engine_parts(s0, s1):
    nf = max(1, s1.frames_done - s0.frames_done)
    return {"steps": s1.steps_done - s0.steps_done,
            "engine_host_ms_per_frame": (s1.host_ms - s0.host_ms) / nf,
            "engine_host_ms_per_frame_by_part": {
                k: (s1.host_stage_ms[i] - s0.host_stage_ms[i]) / nf for i, k in enumerate(
                    ["uploads", "inter", "residual", "intra", "post_filter", "slots_outputs"])},
            "device_ms_per_frame": (s1.device_ms - s0.device_ms) / nf}


def _alone_digests(local, templates, sbs, lengths):
    """Each template decoded alone, as long as its longest stream: the
    per-frame digests every stream of that template must reproduce."""
    from oxideav_av1_b200 import engine
    solo = engine.Engine(device=local, lanes=len(lengths))
    _, dg, _, ok = drive(solo, templates, sbs, [(t, lengths[t]) for t in range(len(templates))],
                         clients=len(templates))
    solo.close()
    # a frame that failed alone is in FRAME_FAILURES, and every stream frame
    # compared with it counts as a mismatch
    return dg


def _host_info():
    return {"host_cpus": len(os.sched_getaffinity(0)), "host_load_avg_1min": os.getloadavg()[0]}


def run_decode(args, local, passes=16):
    """Real AV1 bitstreams end to end: the 110 IVF streams the reference's
    tests/fixture_conformance.rs decodes (carried in
    tests/golden/framing_fixtures.json.gz with the SHA-256 of their decoded
    planes), each through the registry-style stream decoder: the host tile
    walk (symbols, contexts, motion vector prediction) and the GPU engine for
    every pixel stage, whole IVF file in, shown frames out.  8 client threads
    each decode their share of the corpus, `passes` times over, on one
    engine; every stream's digest is checked against the reference's on
    every pass.  The CPU arm decodes the corpus once on one host thread with
    the same walk and the oracle (the C restatement of the reference's pixel
    path).  The streams are small (64x64 to 320x240, 478 shown frames), so
    per-frame fixed costs dominate both arms."""
    import base64
    import gzip
    import threading
    from oxideav_av1_b200 import decoder, engine
    streams = json.load(gzip.open(ROOT / "tests" / "golden" / "framing_fixtures.json.gz"))["ivf_streams"]
    ivfs = [base64.b64decode(x["ivf"]) for x in streams]
    eng = engine.Engine(device=local, lanes=8)
    for b in ivfs[:8]:   # warm-up: pinned pools, memory pool
        decoder.decode(b, eng)
    lock = threading.Lock()
    res = {"frames": 0, "walk_ms": 0.0, "ok": True}

    def client(ids):
        n, walk, ok = 0, 0.0, True
        for _ in range(passes):
            for i in ids:
                dec = decoder.Av1Decoder(eng)
                try:
                    dec.send_packet(ivfs[i])
                    dec.flush()
                    frames = dec.drain()
                    walk += dec.host_ms()
                finally:
                    dec.close()
                ok &= decoder.digest(frames) == streams[i]["sha256"] and len(frames) == streams[i]["shown_frames"]
                n += len(frames)
        with lock:
            res["frames"] += n
            res["walk_ms"] += walk
            res["ok"] &= ok

    # largest streams first, spread over the clients
    order = sorted(range(len(ivfs)), key=lambda i: -len(ivfs[i]))
    threads = [threading.Thread(target=client, args=(order[k::8],)) for k in range(8)]
    t0 = time.perf_counter()
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    wall = time.perf_counter() - t0
    eng.close()
    out = {"streams": len(ivfs), "passes": passes, "frames": res["frames"], "value": res["frames"] / wall,
           "unit": UNIT, "wall_s": wall, "walk_host_ms_per_frame": res["walk_ms"] / max(1, res["frames"]),
           "digests_match_reference": bool(res["ok"]),
           "path": "av1g_decoder_send_packet (whole IVF) / av1g_decoder_receive_frame, one engine, 8 client "
                   "threads", **_host_info()}
    if not args.no_cpu_baseline:
        import oracle
        t0 = time.perf_counter()
        n = 0
        for b in ivfs:
            _, frames = decoder.parse_stream(b)
            n += sum(1 for o in oracle.decode_stream(frames) if o is not None)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"the whole corpus once ({n} shown frames): host walk + oracle, one thread"}
    return out


def mix_templates():
    """The stream-batching mix's templates: every resolution x bit depth (8,
    10) x chroma format (4:2:0, 4:4:4), index = shape * 4 + depth * 2 + format;
    returns (templates, superblock sizes, generation seconds)."""
    specs, sbs = [], []
    for w, h in BATCH_SHAPES:
        for bd in (8, 10):
            for ss in (1, 0):
                sb = 128 if w >= 3840 else 64
                specs.append((900 + len(specs), w, h, bd, ss, False, sb))
                sbs.append(sb)
    t0 = time.perf_counter()
    templates = make_templates(specs)
    return templates, sbs, time.perf_counter() - t0


def _draw_mix_template(rng):
    shape_of = [si for si, wgt in enumerate(BATCH_WEIGHTS) for _ in range(wgt)]
    si = shape_of[int(rng.integers(0, len(shape_of)))]
    return si * 4 + int(rng.integers(0, 2)) * 2 + int(rng.integers(0, 2))


def run_batching(args, local, mix):
    """The stream-batching configuration through the engine: 256 streams of
    uneven shape decoded by the engine batching one frame of every ready
    stream per step (one launch per stage across the streams of a lane)
    against the same engine with one frame per step (the plain per-frame
    launch path), both on the same number of lanes (worker threads with
    their own CUDA streams) and the same 8 client threads, so the ratio is
    the batching alone.  Every stream's output must equal its template
    decoded alone (a CRC-32 of every plane of every frame)."""
    from oxideav_av1_b200 import engine
    rng = np.random.default_rng(11)
    templates, sbs, gen_s = mix
    # stream i: shape by weight, bit depth and chroma format uniform, 8-60 frames
    streams = [(_draw_mix_template(rng), int(rng.integers(8, 61))) for _ in range(args.batch_streams)]
    lengths = [max([n for t_, n in streams if t_ == t] + [1]) for t in range(len(templates))]
    FRAME_FAILURES.clear()
    ref = _alone_digests(local, templates, sbs, lengths)
    frames = sum(n for _, n in streams)
    desc_bytes = sum(_desc_bytes(stream_frame(templates[t], k)) for t, n in streams for k in range(n))
    out = {"streams": len(streams), "frames": frames,
           "mix": "640x360 / 1280x720 / 1920x1080 / 3840x2160 weighted 4:3:2:1, 8- or 10-bit, 4:2:0 or 4:4:4 "
                  "(uniform), 8-60 frames per stream (uniform); 128x128 superblocks and 2 x 2 tiles at 3840x2160",
           "templates": f"{len(templates)} synthetic streams (a key frame with palette blocks, then inter frames with "
                        f"every inter tool, intra blocks and residuals, the post-filter chain); a longer stream "
                        f"cycles its template's inter frames",
           "template_generation_s": gen_s,
           "descriptor_bytes_per_frame": desc_bytes / frames,
           "clients": args.batch_clients,
           "timing": "host wall clock, first submit to last fetch; client threads each owning a group of streams "
                     "(at most 2 frames of a stream in flight); a first run checks a CRC-32 per plane of every "
                     "output frame against the streams decoded alone, two more fetch every frame unhashed and "
                     "the faster is reported",
           **_host_info()}
    # warm-up: every stream for a few frames, so that the engine's pinned
    # pools and the device memory pool reach the run's working set first
    warm = [(t, min(n, 4)) for t, n in streams]
    ok_all = True
    for name, mb in [("batched", 64), ("per_frame", 1)]:
        eng = engine.Engine(device=local, max_batch=mb, lanes=args.serve_lanes)
        drive(eng, templates, sbs, warm, clients=args.batch_clients)
        runs = []
        # run 1 checks every output frame (CRC-32 per plane on the client
        # threads); runs 2 and 3 fetch every frame into host memory without
        # hashing it, so that the check's host work does not compete with the
        # engine's; the faster of those two is reported
        for check in (True, False, False):
            s0 = eng.stats()
            fps, dg, lats, ok = drive(eng, templates, sbs, streams, clients=args.batch_clients, check=check)
            s1 = eng.stats()
            ok_all &= ok
            if check:
                ok_all &= all(d == ref[t][:len(d)] and len(d) == n for d, (t, n) in zip(dg, streams))
            runs.append({"value": fps, "unit": UNIT, "max_frames_per_step": mb, "lanes": args.serve_lanes,
                         "p50_ms": _pct(lats, 0.5), "p99_ms": _pct(lats, 0.99), **_engine_parts(s0, s1)})
        eng.close()
        best = max(runs[1:], key=lambda r: r["value"])
        out[name] = dict(best, checked_run_value=runs[0]["value"], runs_value=[r["value"] for r in runs[1:]])
    out["batched_over_per_frame"] = out["batched"]["value"] / out["per_frame"]["value"]
    out["bit_exact_alone_vs_mixed"] = bool(ok_all)
    out["failed_frames"] = _failures_summary()
    return out


def _desc_bytes(fr):
    """Bytes of one frame's host descriptor (what av1g_submit_frame copies)."""
    n = 0
    for a in [fr.preds, fr.neighbours, fr.warps, fr.inter_tus, fr.intra_tus, fr.coeffs, fr.palette_maps,
              fr.cdef_idx] + list(fr.lr_units or []) + list((fr.grid or {}).values()):
        if a is not None:
            n += np.asarray(a).nbytes
    return n


def _serve_variant(args, local, templates, sbs, draw, mean_len, label):
    """One serving run: closed-loop capacity of the batching engine and of the
    per-frame path (same lanes, budget and clients), then Poisson arrivals at
    30 %, 60 % and 90 % of the batched capacity, and the per-frame path at the
    60 % arrival rate.  A client thread takes each arrival, opens the stream
    (waiting while the budget is full), decodes it with two frames in flight
    and checks every frame against the template decoded alone."""
    import queue
    import threading
    from oxideav_av1_b200 import engine
    rng = np.random.default_rng(17)
    FRAME_FAILURES.clear()
    ref = _alone_digests(local, templates, sbs, [300] * len(templates))
    out = {"what": label, "budget_bytes": SERVE_BUDGET, "lanes": args.serve_lanes,
           "timing": "host wall clock; per-frame latency = the engine's submit-to-completion time", **_host_info()}
    ok_all = True
    cap_streams = [draw(rng) for _ in range(args.serve_cap_streams)]
    for name, mb in [("batched", 64), ("per_frame", 1)]:
        eng = engine.Engine(device=local, max_batch=mb, lanes=args.serve_lanes, budget_bytes=SERVE_BUDGET)
        drive(eng, templates, sbs, [(t, min(n, 6)) for t, n in cap_streams])
        s0 = eng.stats()
        fps, dg, lats, ok = drive(eng, templates, sbs, cap_streams)
        s1 = eng.stats()
        eng.close()
        ok_all &= ok and all(d == ref[t][:n] for d, (t, n) in zip(dg, cap_streams))
        out[f"capacity_{name}"] = {"value": fps, "unit": UNIT, "streams": len(cap_streams),
                                   "frames": sum(n for _, n in cap_streams), "max_frames_per_step": mb,
                                   "p50_ms": _pct(lats, 0.5), "p99_ms": _pct(lats, 0.99), **_engine_parts(s0, s1)}
    cap = out["capacity_batched"]["value"]
    out["stated_rate"] = {"streams_per_s": SERVE_RATE, "offered_frames_per_s": SERVE_RATE * mean_len,
                          "times_batched_capacity": SERVE_RATE * mean_len / cap}

    def poisson(mb, load):
        lam = load * cap / mean_len
        arrivals, t = [], 0.0
        while True:
            t += rng.exponential(1.0 / lam)
            if t > args.serve_seconds:
                break
            arrivals.append((t, draw(rng)))
        eng = engine.Engine(device=local, max_batch=mb, lanes=args.serve_lanes, budget_bytes=SERVE_BUDGET)
        drive(eng, templates, sbs, [(t_, 6) for t_ in range(len(templates))] * 2)
        s0 = eng.stats()
        arrived = queue.Queue()
        lock = threading.Lock()
        res = {"lats": [], "frames": 0, "ok": True, "wait_ms": []}

        def client():
            while True:
                item = arrived.get()
                if item is None:
                    return
                t_arr, (tpl, n) = item
                w0 = time.perf_counter()
                seq = synth.stream_seq(templates[tpl], sbs[tpl])
                hnd = eng.open_stream(seq)
                while hnd is None:  # admitted once the budget frees up
                    time.sleep(0.001)
                    hnd = eng.open_stream(seq)
                wait = (time.perf_counter() - w0) * 1e3
                pend, dg, ls, ok = [], [], [], True
                for k in range(n):
                    if len(pend) >= 2:
                        tk = pend.pop(0)
                        ok &= eng.poll(tk, 300.0) == abi.AV1G_OK
                        st, d, lat = _fetch_digest(eng.lib, hnd.h, tk)
                        ok &= st == abi.AV1G_OK
                        dg.append(d)
                        ls.append(lat)
                    while True:
                        try:
                            pend.append(hnd.submit(stream_frame(templates[tpl], k)))
                            break
                        except abi.Av1gError as e:
                            if e.status != abi.AV1G_EBUSY:
                                raise
                            time.sleep(0.0005)
                for tk in pend:
                    ok &= eng.poll(tk, 300.0) == abi.AV1G_OK
                    st, d, lat = _fetch_digest(eng.lib, hnd.h, tk)
                    ok &= st == abi.AV1G_OK
                    dg.append(d)
                    ls.append(lat)
                hnd.close()
                with lock:
                    res["lats"] += ls
                    res["frames"] += n
                    res["wait_ms"].append(wait)
                    res["ok"] &= ok and dg == ref[tpl][:n]

        threads = [threading.Thread(target=client) for _ in range(args.serve_clients)]
        for th in threads:
            th.start()
        t0 = time.perf_counter()
        for t_arr, item in arrivals:
            d = t0 + t_arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            arrived.put((t_arr, item))
        for _ in threads:
            arrived.put(None)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        s1 = eng.stats()
        eng.close()
        lats = res["lats"]
        return res["ok"], {"load": load, "arrival_rate_streams_per_s": lam, "streams": len(arrivals),
                           "frames": res["frames"], "value": res["frames"] / wall, "unit": UNIT,
                           "wall_s": wall, "p50_ms": _pct(lats, 0.5), "p99_ms": _pct(lats, 0.99),
                           "admission_wait_ms_p99": _pct(res["wait_ms"], 0.99), "max_frames_per_step": mb,
                           **_engine_parts(s0, s1)}

    out["poisson"] = []
    for load in (0.3, 0.6, 0.9):
        ok, r = poisson(64, load)
        ok_all &= ok
        out["poisson"].append(r)
    ok, r = poisson(1, 0.6)
    ok_all &= ok
    out["poisson_per_frame_path"] = r
    out["bit_exact_alone_vs_mixed"] = bool(ok_all)
    out["failed_frames"] = _failures_summary()  # the alone and capacity runs (Poisson runs count in bit_exact)
    return out


def run_serving(args, local, mix):
    """The serving configuration through the engine: Poisson arrivals of
    streams of 30-300 frames (uniform), 25 % with film grain, admitted by a
    120 GB HBM budget; the stated mean rate (40 streams/s) is reported as the
    offered load it is against the measured capacity.  Two stream mixes: the
    batching configuration's resolutions, bit depths and chroma formats, and
    3840x2160 10-bit 4:2:0 only (the full-reconstruction configuration's
    shape)."""
    templates, sbs, gen_s = mix
    # each mix template also with film grain on every frame (index + 16)
    grained = [synth.with_film_grain(t, 77 + i) for i, t in enumerate(templates)]
    mix_t, mix_sb = templates + grained, sbs + sbs

    def draw_mix(rng):
        t = _draw_mix_template(rng) + (len(templates) if rng.random() < 0.25 else 0)
        return t, int(rng.integers(30, 301))

    out = {"mix": _serve_variant(args, local, mix_t, mix_sb, draw_mix, (30 + 300) / 2,
                                 "the batching mix (640x360 / 1280x720 / 1920x1080 / 3840x2160 weighted 4:3:2:1, "
                                 "8- or 10-bit, 4:2:0 or 4:4:4), 30-300 frames per stream, 25 % with film grain")}
    w, h, bd = SERVE_SHAPE
    specs = [(950 + i, w, h, bd, 1, grain, 128) for i, grain in enumerate([False, False, True, True])]
    t0 = time.perf_counter()
    uhd = make_templates(specs)
    gen_uhd = time.perf_counter() - t0

    def draw_uhd(rng):
        grain = rng.random() < 0.25
        return (2 if grain else 0) + int(rng.integers(0, 2)), int(rng.integers(30, 301))

    out["uhd"] = _serve_variant(args, local, uhd, [128] * len(uhd), draw_uhd, (30 + 300) / 2,
                                f"{w}x{h} {bd}-bit 4:2:0, 128x128 superblocks, 2 x 2 tiles, 30-300 frames per "
                                f"stream, 25 % with film grain")
    out["template_generation_s"] = gen_s + gen_uhd
    return out


def run_e2e(args, frames, dframes, jobs, stream, dev, world, chunks=8, graphs=True):
    """Frames/s through the C-ABI with host buffers: every step copies all
    inputs from pinned host memory, runs the chain and copies the restored
    (cropped) planes back.  The batch is cut into `chunks` groups of frames so
    that the copies of one group overlap the kernels of the next (three CUDA
    streams: host-to-device, compute, device-to-host), the way a serving loop
    feeds the engine; every byte is still copied every step.  Each group's
    chain runs through av1g_run_postfilter, which validates and prepares the
    group's frame records on the host every call and stores them with small
    kernel launches (no copy engine, so they never queue behind the large
    input copies); graphs=True instead captures each group's chain once as a
    CUDA graph (av1g_chain_graph_create over the group's buffers) and replays
    it per step (av1g_chain_graph_launch)."""
    import torch
    from oxideav_av1_b200 import postfilter

    lib = abi.load()
    n = len(dframes)
    per = (n + chunks - 1) // chunks
    groups = [list(range(c * per, min(n, (c + 1) * per))) for c in range(chunks) if c * per < n]

    def arena(tensors):
        """Moves the tensors into views of one device buffer (256-byte aligned
        offsets), so that a group's inputs or outputs cross PCIe as one copy."""
        offs, total = [], 0
        for t in tensors:
            offs.append(total)
            total = (total + t.numel() * t.element_size() + 255) // 256 * 256
        buf = torch.empty(total, dtype=torch.uint8, device=dev)
        views = []
        for t, o in zip(tensors, offs):
            v = buf[o:o + t.numel() * t.element_size()].view(t.dtype).view(t.shape)
            v.copy_(t)
            views.append(v)
        return buf, views

    h_in, d_in, h_out, d_out = [], [], [], []
    for g in groups:
        ins, outs = [], []
        for i in g:
            d = dframes[i]
            ins += [pl.t for pl in d.recon] + [d.grid[k] for k in d.GRID_KEYS] + [d.cdef_idx]
            ins += [u for u in d.lr_units if u is not None]
            outs += [pl.t for pl in d.stage_planes()["lr"]]
        buf_in, vin = arena(ins)
        buf_out, vout = arena(outs)
        it_in, it_out = iter(vin), iter(vout)
        for i in g:       # re-point the frames at the arena views, in the same order
            d = dframes[i]
            for pl in d.recon:
                pl.t = next(it_in)
            for k in d.GRID_KEYS:
                d.grid[k] = next(it_in)
            d.cdef_idx = next(it_in)
            d.lr_units = [next(it_in) if u is not None else None for u in d.lr_units]
            for pl in d.stage_planes()["lr"]:
                pl.t = next(it_out)
        d_in.append(buf_in)
        d_out.append(buf_out)
        h_in.append(buf_in.cpu().pin_memory())
        h_out.append(torch.empty_like(buf_out, device="cpu").pin_memory())
    gjobs = [postfilter.jobs_array([dframes[i] for i in g]) for g in groups]
    sp = C.c_void_p(stream.cuda_stream)
    ggraph = []
    if graphs:  # each group's chain captured once over its arena-backed frames
        for gi, g in enumerate(groups):
            gh = C.c_void_p()
            abi.check(lib.av1g_chain_graph_create(gjobs[gi], len(g), (1 << 5) - 1, abi.MODE_BATCHED, sp,
                                                  C.byref(gh)))
            ggraph.append(gh)
    s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    h2d = sum(t.numel() for t in h_in)
    d2h = sum(t.numel() for t in h_out)

    ev_comp = [torch.cuda.Event() for _ in groups]   # group's kernels done (inputs free)
    ev_d2h = [torch.cuda.Event() for _ in groups]    # group's outputs copied out (outputs free)
    ev_in = [torch.cuda.Event() for _ in groups]
    call_s = [0.0, 0]  # host seconds inside the library's entry point, calls

    def step():
        for gi in range(len(groups)):
            with torch.cuda.stream(s_in):
                s_in.wait_event(ev_comp[gi])
                d_in[gi].copy_(h_in[gi], non_blocking=True)
                ev_in[gi].record(s_in)
            stream.wait_event(ev_in[gi])
            stream.wait_event(ev_d2h[gi])
            t0 = time.perf_counter()
            if graphs:
                rc = lib.av1g_chain_graph_launch(ggraph[gi], sp)
            else:
                rc = lib.av1g_run_postfilter(gjobs[gi], len(groups[gi]), abi.MODE_BATCHED, sp, None)
            call_s[0] += time.perf_counter() - t0
            call_s[1] += 1
            abi.check(rc)
            ev_comp[gi].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_comp[gi])
                h_out[gi].copy_(d_out[gi], non_blocking=True)
                ev_d2h[gi].record(s_out)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    call_s[0], call_s[1] = 0.0, 0
    h0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    stream.wait_stream(s_out)
    e1.record(stream)
    host_ms = (time.perf_counter() - h0) * 1e3 / args.steps
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
    host = {"enqueue_ms_per_step": host_ms, "entry_point_ms_per_call": call_s[0] * 1e3 / max(call_s[1], 1),
            "calls_per_step": len(groups),
            "note": "host wall time to enqueue one step (all groups' copies, chain calls and events) and the "
                    "mean host time inside the library call; enqueue time near ms_per_step means the step is "
                    "bound by the host, not the GPU"}
    for gh in ggraph:
        abi.check(lib.av1g_chain_graph_destroy(gh))

    def copies_ms(h2d_on, d2h_on, reps=3):
        """The step's copies alone, on the same pinned buffers and streams:
        the PCIe floor the end-to-end step can approach."""
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        s_in.wait_event(c0)
        s_out.wait_event(c0)
        for _ in range(reps):
            for gi in range(len(groups)):
                if h2d_on:
                    with torch.cuda.stream(s_in):
                        d_in[gi].copy_(h_in[gi], non_blocking=True)
                if d2h_on:
                    with torch.cuda.stream(s_out):
                        h_out[gi].copy_(d_out[gi], non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        c1.record(stream)
        torch.cuda.synchronize()
        return c0.elapsed_time(c1) / reps

    t_in, t_out, t_both = copies_ms(True, False), copies_ms(False, True), copies_ms(True, True)
    pcie = {"h2d_gbs": h2d / t_in / 1e6, "d2h_gbs": d2h / t_out / 1e6, "both_ms_per_step": t_both,
            "floor_ms_per_step": max(t_in, t_out, t_both),
            "e2e_frac_of_floor": max(t_in, t_out, t_both) / ms,
            "note": "the step's pinned copies alone (same buffers and streams, no kernels): h2d and d2h each "
                    "alone, then both at once; floor = the slowest of the three"}
    return {"value": job_rate(world, n, ms), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms, "pcie": pcie, "host": host,
            "path": f"{'av1g_chain_graph_launch (one captured chain per group)' if graphs else 'av1g_run_postfilter'}"
                    f" with pinned-host inputs/outputs copied every step, {len(groups)} groups of frames (one copy "
                    f"in and one copy out per group) pipelined over copy-in / compute / copy-out streams"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=64)
    ap.add_argument("--bit-depth", type=int, default=8, choices=[8, 10])
    ap.add_argument("--cpu-sample", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--batch-streams", type=int, default=256)
    ap.add_argument("--batch-clients", type=int, default=8)
    ap.add_argument("--serve-cap-streams", type=int, default=12)
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-clients", type=int, default=32)
    ap.add_argument("--serve-lanes", type=int, default=8)
    ap.add_argument("--section", default="all",
                    choices=["all", "recon", "extra", "motion_field", "chain", "e2e", "decode", "batching",
                             "serving"],
                    help="recon / extra: only that section (one GPU), printed as its own JSON object; "
                         "for profiling a row's kernels")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.section != "all":
        import torch
        torch.cuda.set_device(0)
        abi.load()
        if args.section == "decode":
            print(json.dumps({"decode": run_decode(args, 0)}), flush=True)
            return 0
        if args.section in ("batching", "serving"):
            fn = run_batching if args.section == "batching" else run_serving
            print(json.dumps({args.section: fn(args, 0, mix_templates())}), flush=True)
            return 0
        stream = torch.cuda.Stream()
        fn = {"chain": run_chain, "e2e": run_e2e_section, "recon": run_recon_stages, "extra": run_extra_stages,
              "motion_field": run_motion_field}[args.section]
        print(json.dumps({args.section: fn(args, torch.device("cuda", 0), stream)}), flush=True)
        return 0
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
