#!/usr/bin/env python
"""Benchmark of the TGMM supervoxel VI-EM on B200: EM frames/s on the 1-Gvoxel frame
(2048x1024x512, 20,000 nuclei, 5 candidates, 20 iterations), with voxel-iterations/s,
per-frame latency percentiles, the roofline of the per-iteration voxel pass, an
end-to-end figure through the C ABI with host buffers, and the CPU baseline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one EM call (20 iterations) over one synthetic frame.  With N GPUs every
rank runs its own frame (replicas: frames are independent, no collective on the data
path) and `value` is the whole-job frames/s.  `--impl reference` times the reference's
CPU arithmetic (the FP32 OpenMP port of its kernels in oracle/) on the host cores.
"""
from __future__ import annotations

import argparse
import datetime
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

METRIC = "EM frames/s & voxel-iters/s at 1 Gvox/20k nuclei; p50/p99 frame latency"
UNIT = "frames/s"
WORKLOAD = "2048x1024x512 uint16 volume, 20000 nuclei (semi-axes 4-8, anisotropy 2), 5-NN, 20 EM iterations"
EM_ITERS = 20
# kernels the engine launches per EM call: build_maps, import, moments,
# 4 per iteration (knn_estep, mstep_update, kill_prep, ll_pass),
# assign, export
KERNELS_PER_CALL = 3 + 4 * EM_ITERS + 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["c2", "c1"], default="c2")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=2000)
    return ap.parse_args()


def spec_for(name):
    from tgmm_b200 import synth
    return synth.C2 if name == "c2" else synth.C1


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes (read + write) per launch of the voxel pass from the committed ncu summary,
    with the voxel count of the captured frame, or None.  The pass streams each voxel once,
    so its traffic scales with the voxel count."""
    p = os.path.join(ROOT, "profiles", "ll_pass_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_setup(backend):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def cpu_baseline(frame, threads=None):
    """The reference's FP32 kernel arithmetic (oracle REF32 port) on the host cores, one EM
    iteration of the workload frame as the bounded sample, scaled to 20 iterations."""
    from oracle import oracle as O
    n = threads or os.cpu_count() or 1
    O.lib().or_set_num_threads(n)
    p = O.params(max_iter=1, tol=-1.0, mode=O.MODE_REF32)
    t0 = time.perf_counter()
    O.em_run(frame.query, frame.img, frame.centroids, frame.label_ptr, frame.gauss, p)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / (EM_ITERS * dt), "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"1 of {EM_ITERS} EM iterations of the workload frame with the FP32 OpenMP port of the "
                      f"reference kernels ({dt:.2f} s), scaled to {EM_ITERS} iterations"}, dt


def run_reference(args):
    world, rank, local = dist_setup("gloo")
    if rank != 0:
        return
    from tgmm_b200 import synth
    spec = spec_for(args.workload)
    frame = synth.generate(spec, seed=args.seed)
    times = []
    info = None
    for i in range(args.warmup + args.steps):
        info, dt = cpu_baseline(frame)
        if i >= args.warmup:
            times.append(dt)
    per_frame = EM_ITERS * float(np.sum(times)) / len(times)
    value = 1.0 / per_frame
    info["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_frame * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_vox": frame.n_vox, "n_sv": frame.n_sv, "n_gauss": frame.n_gauss},
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    from tgmm_b200 import synth

    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = spec_for(args.workload)
    frame = synth.generate(spec, seed=args.seed + rank)  # each replica its own frame
    params = synth.em_params(iters=EM_ITERS, tol=-1.0)
    df = E.to_device(frame, dev)
    gm0 = E.gauss_to_device(frame.gauss, dev)
    gm = gm0.clone()
    S, K, N = frame.n_sv, frame.n_gauss, frame.n_vox
    rnk = torch.empty(5 * S, dtype=torch.float32, device=dev)
    ind = torch.empty(5 * S, dtype=torch.int32, device=dev)
    plan = E.Plan(N, S, K, device=local)
    stream = torch.cuda.current_stream(dev)

    def step():
        gm.copy_(gm0, non_blocking=True)
        plan.run_device(df, gm, rnk, ind, params, stats=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    check = plan.run_device(df, gm.copy_(gm0), rnk, ind, params, stats=True)
    assert check["iterations"] == EM_ITERS, check

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        ev[0].record(stream)
        for i in range(args.steps):
            step()
            ev[i + 1].record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    nv = torch.tensor([float(N)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(nv, op=dist.ReduceOp.SUM)
    max_ms = float(t.item())
    total_vox = float(nv.item())
    value = world * args.steps / (max_ms / 1e3)
    voxel_iters = total_vox * EM_ITERS * args.steps / (max_ms / 1e3)

    # roofline of the per-iteration voxel pass (timed alone on this stream, same workload)
    ms_ll = plan_time(plan, L.TGMM_KERNEL_LL_PASS, 20, stream)
    ms_mom = plan_time(plan, L.TGMM_KERNEL_MOMENTS, 10, stream)
    peak, peak_kind = measured_peaks()
    alg_bytes = 16.0 * N
    achieved = alg_bytes / (ms_ll * 1e-3) / 1e9
    traffic = committed_traffic()
    roofline = {"bound": "hbm", "kernel": "k_ll_pass (log-likelihood voxel pass, per iteration)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else
                "fallback 6650 GB/s", "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": ms_ll,
                "traffic": (traffic["bytes_per_launch"] * N / traffic["n_vox"]) if traffic else None,
                "moments_pass": {"ms_per_launch": ms_mom, "achieved": alg_bytes / (ms_mom * 1e-3) / 1e9,
                                 "frac": alg_bytes / (ms_mom * 1e-3) / 1e9 / peak}}

    # end to end through the C ABI with host buffers: H2D of the frame, Gaussians H2D/D2H
    # inside tgmm_em_run, D2H of rnk/ind, every step
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(frame, df, plan, params, dev, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = cpu_baseline(frame)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "n_vox": N, "n_sv": S, "n_gauss": K, "em_iterations": EM_ITERS,
                           "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (16 B x n_vox)",
                           "ll_precision": "mixed", "ll_mode": "as_reference"},
                "voxel_iters_per_s": voxel_iters,
                "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
                "gpu_launches": KERNELS_PER_CALL * args.steps,
                "roofline": roofline, "clocks": clocks.summary(), "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def plan_time(plan, kernel, reps, stream):
    import ctypes as C
    from tgmm_b200 import _lib as L
    ms = C.c_float()
    L.check(L.gmem().tgmm_plan_time_kernel(plan.h, kernel, reps, C.byref(ms), stream.cuda_stream),
            "tgmm_plan_time_kernel")
    return float(ms.value)


def run_e2e(frame, df, plan, params, dev, args):
    import ctypes as C
    import torch
    from tgmm_b200 import _lib as L
    pin = {k: torch.from_numpy(np.ascontiguousarray(getattr(frame, k))).pin_memory()
           for k in ("query", "img", "centroids", "label_ptr")}
    S, K = frame.n_sv, frame.n_gauss
    rnk_h = torch.empty(5 * S, dtype=torch.float32).pin_memory()
    ind_h = torch.empty(5 * S, dtype=torch.int32).pin_memory()
    rnk = torch.empty(5 * S, dtype=torch.float32, device=dev)
    ind = torch.empty(5 * S, dtype=torch.int32, device=dev)
    g_host = np.ascontiguousarray(frame.gauss.astype(L.GAUSS_DTYPE))
    stream = torch.cuda.current_stream(dev)
    st = L.TgmmEmStats()
    lib = L.gmem()
    h2d = sum(int(v.numel() * v.element_size()) for v in pin.values()) + 288 * K
    d2h = 288 * K + 8 * 5 * S

    def one():
        g = g_host.copy()
        df.query.copy_(pin["query"], non_blocking=True)
        df.img.copy_(pin["img"], non_blocking=True)
        df.centroids.copy_(pin["centroids"], non_blocking=True)
        df.label_ptr.copy_(pin["label_ptr"], non_blocking=True)
        cf = df.cframe()
        L.check(lib.tgmm_em_run(plan.h, C.byref(cf), g.ctypes.data, rnk.data_ptr(), ind.data_ptr(), None,
                                C.byref(params), C.byref(st), stream.cuda_stream), "tgmm_em_run")
        rnk_h.copy_(rnk, non_blocking=True)
        ind_h.copy_(ind, non_blocking=True)
        torch.cuda.synchronize(dev)
        return g

    for _ in range(max(1, args.warmup)):
        one()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    a.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    b.record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    ms = a.elapsed_time(b)
    return {"value": args.steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "wall_frames_per_s": args.steps / wall, "path": "tgmm_em_run (C ABI) with pinned host buffers"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
