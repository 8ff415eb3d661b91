"""Benchmark: MPix/s of the full two-step GBM3D on a 4096 x 4096 image, sigma 25.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full GBM3D denoise (source/GBM3D.m, 'default' profile: step-1
matching + global 3D bior1.5 x Haar hard thresholding + aggregation over two
match spins, then step-2 matching + empirical Wiener + aggregation over two
match spins) of one synthetic 4096^2 image resident in HBM.  Under torchrun
every rank denoises its own image on its own GPU (independent images: weak
scaling, no collective on the data path); the time is the max over ranks.

--impl reference times the CPU restatement of the reference path (the oracle,
all host threads) on bounded crops of the same workload.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MPix/s 2-step GBM3D at 4096^2, sigma=25 (plain path)"
SIZE = 4096
SIGMA = 25.0
PROFILE = "default"
WORKLOAD = ("GBM3D 'default' profile (blockSize 16 / blockSizeWie 8, matchSize 32, numMax 16, "
            "match spins [0 4] + [0 4], 2 cycle spins, bior1.5 x Haar, 3 levels) on one "
            "4096x4096 synthetic image, sigma 25, float64 in/out")


def _set_size(size: int) -> None:
    global SIZE, WORKLOAD
    if size != SIZE:
        WORKLOAD = WORKLOAD.replace(f"{SIZE}x{SIZE}", f"{size}x{size}")
        SIZE = size


def _config(extra=None):
    c = {"workload": WORKLOAD, "image": [SIZE, SIZE], "sigma": SIGMA, "profile": PROFILE,
         "parallelism": "replicas: one image per GPU",
         "l2": "inputs larger than L2: each step streams ~10 GB of intermediates through HBM"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4)
                          if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def cpu_baseline(size: int = 1024):
    """The oracle (FP32 restatement of the reference path) on a bounded crop, all host threads."""
    from gbm3d_b200 import options, synth
    from oracle import oracle as O
    O.lib()
    _, noisy = synth.noisy_image(size, size, SIGMA, seed=2024)
    opts = options.resolve_opts({"profile": PROFILE})
    t0 = time.perf_counter()
    O.GBM3D(noisy, SIGMA, opts, prec=32)
    dt = time.perf_counter() - t0
    return {"value": size * size / 1e6 / dt, "unit": "MPix/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"one {size}x{size} crop of the same synthetic workload, FP32 oracle, OpenMP",
            "seconds": dt}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    size = args.ref_size
    base = cpu_baseline.__wrapped__ if hasattr(cpu_baseline, "__wrapped__") else None  # noqa: F841
    from gbm3d_b200 import options, synth
    from oracle import oracle as O
    O.lib()
    _, noisy = synth.noisy_image(size, size, SIGMA, seed=2024)
    opts = options.resolve_opts({"profile": PROFILE})
    for _ in range(args.warmup):
        O.GBM3D(noisy, SIGMA, opts, prec=32)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.GBM3D(noisy, SIGMA, opts, prec=32)
        times.append(time.perf_counter() - t0)
    per = sum(times) / len(times)
    v = size * size / 1e6 / per
    line = {"metric": METRIC, "value": v, "unit": "MPix/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per * 1e3 * (SIZE * SIZE) / (size * size),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": _config({"sample": f"{size}x{size} crop per step"}),
            "cpu_baseline": {"value": v, "unit": "MPix/s", "cores": O.num_threads(), "kind": "port",
                             "sample": f"{size}x{size} crop of the 4096^2 synthetic workload per step, "
                                       "FP32 CPU restatement of the reference path, OpenMP on all host threads"},
            "e2e": {"value": v, "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from gbm3d_b200 import _lib, api, build, synth
    build.build()
    ctx = _lib.Context(local)
    # an explicit stream shared by the library and the timing events (torch's
    # default stream is the legacy NULL stream, which the library's own
    # non-blocking stream does not order against)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    _, noisy = synth.noisy_image(SIZE, SIZE, SIGMA, seed=100 + rank)
    dI = torch.from_numpy(np.asfortranarray(noisy).ravel(order="F")).to(dev)
    dU = torch.empty_like(dI)

    def step():
        api.GBM3D_device(dI.data_ptr(), SIZE, SIZE, SIGMA, dU.data_ptr(), {"profile": PROFILE}, ctx=ctx)

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    launches = ctx.launch_count()

    # per-stage device times from one extra untimed step
    ctx.enable_timing(True)
    step()
    torch.cuda.synchronize()
    stages = ctx.stage_times()
    ctx.enable_timing(False)

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    mpix = SIZE * SIZE / 1e6
    value = world * mpix / (ms / 1e3)

    # end to end through the public host API: pinned host input, H2D + compute + D2H every step
    hI = torch.from_numpy(np.asfortranarray(noisy).ravel(order="F")).pin_memory()
    hU = torch.empty_like(hI).pin_memory()
    import ctypes as C
    co = api.c_opts(api._opt.resolve_opts({"profile": PROFILE}))

    def e2e_step():
        ctx.check(_lib.lib().gbm3d_denoise(ctx.h, C.c_void_p(hI.data_ptr()), SIZE, SIZE, SIGMA, C.byref(co),
                                           C.c_void_p(hU.data_ptr()), None))

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    err = float(np.max(np.abs(hU.numpy().reshape(SIZE, SIZE, order="F") - dU.cpu().numpy().reshape(SIZE, SIZE, order="F"))))

    # roofline of the dominant kernel: step-1 block matching (FP32 CUDA cores)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    n_ref1 = (SIZE // 16) ** 2
    flop1 = n_ref1 * 32 * 32 * 16 * 16 * 3  # N_ref * W^2 * d^2 * 3 (sub, mul, add)
    n_ref2 = (SIZE // 8) ** 2
    flop2 = n_ref2 * 32 * 32 * 8 * 8 * 3
    match1_ms = stages[1] / 2 if len(stages) > 1 else None  # two match spins
    sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s, FMA = 2 flop
    roof = None
    if match1_ms:
        ach = flop1 / (match1_ms / 1e3) / 1e12
        roof = {"kernel": "k_match<16,32> (step-1 block matching)", "bound": "fp32", "achieved": ach,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak, "traffic": None,
                "peak_source": "derived: 148 SMs x 128 FP32 lanes x 2 flop x median SM clock under load "
                               "(MEASURED_PEAKS.json has no FP32 SIMT figure)",
                "algorithmic": f"{flop1 / 1e9:.1f} GFLOP per launch (N_ref*W^2*d^2*3)"}
    line = {"metric": METRIC, "value": value, "unit": "MPix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": _config(),
            "clocks": clk,
            "e2e": {"value": world * mpix / (e2e_ms / 1e3), "unit": "MPix/s",
                    "h2d_bytes_per_step": int(hI.numel() * 8), "d2h_bytes_per_step": int(hU.numel() * 8),
                    "ms_per_step": e2e_ms, "max_abs_vs_device_path": err},
            "gpu_launches": launches * args.steps,
            "stages_ms": dict(zip(["glue", "match1", "wavelet1", "agg1", "match2", "wiener2", "agg2", "total"],
                                  stages)),
            "roofline": roof,
            "flop_per_step": {"match1": 2 * flop1, "match2": 2 * flop2}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_size)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-size", type=int, default=1024)
    ap.add_argument("--ref-size", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", type=int, default=SIZE, help="image side (profiling runs use smaller images)")
    args = ap.parse_args()
    _set_size(args.size)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
