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
WORKLOADS = {"c2": WORKLOAD,
             "c1": "256x256x64 uint16 volume, 300 nuclei (semi-axes 3-6, anisotropy 2), 5-NN, 20 EM iterations"}
EM_ITERS = 20


def kernels_per_call(knn_fused: bool) -> int:
    """Kernels the engine launches per EM call: 3 table stagings (k_stage), build_maps, the
    records' fetch and import, the 3 order kernels (sv_records, order_base, order_scatter), the
    moment pass, the first iteration's knn_estep, 3 per iteration (mstep_update, kill_prep,
    ll_pass), the later iterations' knn_estep unless the voxel pass runs them, assign, export
    (a fixed iteration count: no conditional iterations)."""
    return 3 + 8 + 3 * EM_ITERS + (0 if knn_fused else EM_ITERS - 1) + 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["c2", "c1", "batch64", "series", "mixed", "frames"], default="c2",
                    help="c2: the 1-Gvoxel frame (default, the headline); c1: 256x256x64; batch64: 64 uneven "
                         "volumes in one batched call vs one at a time; series: one served time series of "
                         "1024x1024x256 frames; mixed: four served time series of four sizes vs the plain form; "
                         "frames: frame preparation (trimming, centroids, rescale, SoA/CSR) of the c2 volume "
                         "from its raw image and label volume")
    ap.add_argument("--fb-dims", default="", help="frames: X,Y,Z of a smaller volume (profiling)")
    ap.add_argument("--fb-nuclei", type=int, default=0, help="frames: nuclei of the --fb-dims volume")
    ap.add_argument("--frames", type=int, default=0, help="frames per time series (series/mixed; 0 = default sample)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=2000)
    ap.add_argument("--knn-lanes", type=int, choices=[4, 8, 16, 32], default=0,
                    help="fix the kNN/E-step width instead of autotuning (with --knn-fused; for profiling)")
    ap.add_argument("--knn-fused", type=int, choices=[0, 1], default=0,
                    help="with --knn-lanes: 1 = the voxel pass runs the next iteration's kNN/E-step")
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


def committed_traffic(kernel):
    """DRAM bytes (read + write) per launch of the voxel pass (the form named `kernel`) from
    the committed ncu summary, with the voxel count of the captured frame, or None.  The pass
    streams each voxel once, so its traffic scales with the voxel count."""
    p = os.path.join(ROOT, "profiles", "ll_pass_traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)
        return t if t.get("kernel") == kernel else None
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


def reduce_job(total_ms, n_vox, steps, world, device):
    """Whole-job figures from every rank's device time: the slowest rank's time, the voxels
    of all ranks (each rank runs its own frame).  Returns (frames/s, voxel-iterations/s,
    max ms, total voxels)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
    nv = torch.tensor([float(n_vox)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(nv, op=dist.ReduceOp.SUM)
    max_ms = float(t.item())
    total_vox = float(nv.item())
    return world * steps / (max_ms / 1e3), total_vox * EM_ITERS * steps / (max_ms / 1e3), max_ms, total_vox


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(frame, threads=None, single=False):
    """The reference's FP32 kernel arithmetic (the oracle's REF32 port, OpenMP over the host
    cores) on the workload frame: one whole EM call, the same 20 iterations the GPU runs, as
    the bounded sample; with `single`, one iteration of it on one thread, for context."""
    from oracle import oracle as O
    n = threads or os.cpu_count() or 1
    O.lib().or_set_num_threads(n)
    t0 = time.perf_counter()
    out = O.em_run(frame.query, frame.img, frame.centroids, frame.label_ptr, frame.gauss,
                   O.params(max_iter=EM_ITERS, tol=-1.0, mode=O.MODE_REF32))
    dt = time.perf_counter() - t0
    assert out["iterations"] == EM_ITERS
    info = {"value": 1.0 / dt, "unit": UNIT, "cores": n, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"one whole EM call ({EM_ITERS} iterations) of the workload frame with the FP32 OpenMP port "
                      f"of the reference kernels ({dt:.2f} s)"}
    if single:
        O.lib().or_set_num_threads(1)
        t0 = time.perf_counter()
        O.em_run(frame.query, frame.img, frame.centroids, frame.label_ptr, frame.gauss,
                 O.params(max_iter=1, tol=-1.0, mode=O.MODE_REF32))
        d1 = time.perf_counter() - t0
        O.lib().or_set_num_threads(n)
        info["single_thread"] = {"value": 1.0 / (EM_ITERS * d1), "unit": UNIT, "cores": 1,
                                 "sample": f"one of the {EM_ITERS} iterations on one thread ({d1:.2f} s), "
                                           f"scaled to {EM_ITERS}"}
    return info, dt


PARITY_TOL = {"rnk_max_abs": 1e-5, "m_max_abs_voxel": 1e-3, "w_max_rel": 1e-4, "ll_rel": 1e-6}


def parity_vs_oracle(frame, got):
    """The GPU call's outputs (got: gauss records, rnk, ind, ll) against the FP64 oracle's
    EM on the same frame and parameters: kNN candidates and supervoxel assignments exact,
    the largest errors of rnk, means, precision matrices (relative to the largest entry of
    each) and log-likelihood beside their tolerances.  Outside every timed region."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    o = O.em_run(frame.query, frame.img, frame.centroids, frame.label_ptr, frame.gauss,
                 O.params(max_iter=EM_ITERS, tol=-1.0))
    dt = time.perf_counter() - t0
    gg, og = got["gauss"], o["gauss"]
    a = og["m_o"][:, 0] > -1e31
    wscale = np.max(np.abs(og["W_k"][a]), axis=1, keepdims=True)
    assign = bool(np.array_equal(gg["supervoxelNum"], og["supervoxelNum"]) and all(
        np.array_equal(gg["supervoxelIdx"][k][:og["supervoxelNum"][k]], og["supervoxelIdx"][k][:og["supervoxelNum"][k]])
        for k in range(og.shape[0])))
    err = {"ind_equal": bool(np.array_equal(got["ind"], o["ind"])), "assignments_equal": assign,
           "alive_equal": bool(np.array_equal(gg["m_o"][:, 0] > -1e31, a)),
           "rnk_max_abs": float(np.max(np.abs(got["rnk"] - o["rnk"]))),
           "m_max_abs_voxel": float(np.max(np.abs(gg["m_k"][a] - og["m_k"][a]))),
           "w_max_rel": float(np.max(np.abs(gg["W_k"][a] - og["W_k"][a]) / wscale)),
           "ll_rel": abs(got["ll"] - o["ll"]) / abs(o["ll"])}
    err["within_tolerance"] = bool(err["ind_equal"] and err["assignments_equal"] and err["alive_equal"] and
                                   all(err[k] <= v for k, v in PARITY_TOL.items()))
    err["tolerance"] = PARITY_TOL
    err["oracle"] = f"FP64 CPU oracle, {EM_ITERS} iterations, {os.cpu_count()} threads ({dt:.1f} s)"
    return err


def reference_gpu(frame, reps=3):
    """The reference's own GPU path (GMEMvariationalInferenceCUDAWithSupervoxels compiled from
    its sources for sm_100a) on the workload frame, per synchronous call with host arrays in
    and out as its callers use it (its context creation, allocations and copies included).
    Its kNN kernel returns early for the surplus threads of its last block before a
    __syncthreads(), well-defined only when no thread of a block leaves: a frame above 1024
    supervoxels runs padded to a multiple of 1024 with empty supervoxels, which leaves the real
    supervoxels' outputs unchanged (checked on the C1 frame by tests/test_gpu_reference.py)."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "oracle/_ref/libtgmm_ref.so not built (the reference sources were absent)"}
    cent, lptr, padded = frame.centroids, frame.label_ptr, 0
    if frame.n_sv > 1024:
        cent, lptr = O.pad_supervoxels(frame.centroids, frame.label_ptr)
        padded = lptr.shape[0] - 1 - frame.n_sv
    try:
        O.ref_em_run(frame.query, frame.img, cent, lptr, frame.gauss, max_iter=EM_ITERS)  # warm
    except (OSError, RuntimeError) as e:
        return {"unavailable": f"the reference's GPU path did not run: {str(e).splitlines()[0]}"}
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.ref_em_run(frame.query, frame.img, cent, lptr, frame.gauss, max_iter=EM_ITERS)
        ts.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.median(ts))
    return {"value": 1e3 / ms, "unit": UNIT, "ms_per_call": ms, "calls": reps, "padded_supervoxels": padded,
            "path": "the reference's GPU path compiled from its sources, host arrays in and out, per call"}


def fb_spec(args):
    from tgmm_b200 import synth
    if args.fb_dims:
        dims = tuple(int(x) for x in args.fb_dims.split(","))
        return synth.VolumeSpec(dims=dims, n_nuclei=args.fb_nuclei or max(1, dims[0] * dims[1] * dims[2] // 53687),
                                axis_min=4.0, axis_max=8.0)
    return synth.C2


def run_reference_frames(args):
    """The reference arm of the frame-preparation workload: the reference's host build, as the
    oracle's single-thread C restatement, on the same volume; each step one whole volume."""
    import torch
    from oracle import oracle as O
    spec = fb_spec(args)
    raw, lab, S, Nfg, _, _ = fb_volume(spec, args.seed, torch.device("cpu"))
    X, Y, Z = spec.dims
    raw_n = raw.numpy().view(np.uint16).reshape(Z, Y, X)
    lab_n = lab.numpy().view(np.uint32).reshape(Z, Y, X)
    kind = "reference" if O.ref_f1_available() else "port"
    if kind == "reference":  # the supervoxels as the reference holds them: sorted pixel lists
        lists = O.supervoxel_lists(lab_n, S)
    times = []
    out = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if kind == "reference":
            rc, out = O.ref_frame_build(raw_n, lab_n, S, max_vox=Nfg, lists=lists)
        else:
            rc, out = O.frame_build(raw_n, lab_n, S, max_vox=Nfg)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
        assert rc == 0
    per = float(np.mean(times))
    value = 1.0 / per
    if kind == "reference":
        sample = (f"the whole {X}x{Y}x{Z} volume per step: the tracking program's host build loop with the "
                  f"reference's own trimSupervoxel, weightedGaussianStatistics and erase compiled from its sources, "
                  f"one thread ({per:.2f} s)")
    else:
        sample = (f"the whole {X}x{Y}x{Z} volume per step through the oracle's single-thread C restatement of the "
                  f"reference's host build ({per:.2f} s)")
    line = {"impl": "reference", "metric": "frame preparations/s", "value": value, "unit": "volumes/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16/u32 -> f32",
            "data": "synthetic (seeded nuclei volume; labels = its supervoxels)",
            "config": {"workload": f"frame preparation of a {X}x{Y}x{Z} uint16 volume with {S} labelled "
                                   f"supervoxels ({Nfg} labelled voxels): trim, erase, centroids, background, "
                                   f"[0,1] rescale, SoA/CSR", "n_vox_out": out["n_vox"], "n_sv_out": out["n_sv"]},
            "cpu_baseline": {"value": value, "unit": "volumes/s", "cores": 1, "kind": kind, "cpu_model": cpu_model(),
                             "sample": sample},
            "e2e": {"value": value, "unit": "volumes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    world, rank, local = dist_setup("gloo")
    if rank != 0:
        return
    if args.workload == "frames":
        run_reference_frames(args)
        return
    from oracle import oracle as O
    from tgmm_b200 import synth
    spec = spec_for(args.workload)
    frame = synth.generate(spec, seed=args.seed)
    n = os.cpu_count() or 1
    O.lib().or_set_num_threads(n)
    p = O.params(max_iter=EM_ITERS, tol=-1.0, mode=O.MODE_REF32)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = O.em_run(frame.query, frame.img, frame.centroids, frame.label_ptr, frame.gauss, p)
        dt = time.perf_counter() - t0
        assert out["iterations"] == EM_ITERS
        if i >= args.warmup:
            times.append(dt)
    per_frame = float(np.mean(times))
    value = 1.0 / per_frame
    info = {"value": value, "unit": UNIT, "cores": n, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"each step one whole EM call ({EM_ITERS} iterations) of the workload frame with the FP32 "
                      f"OpenMP port of the reference kernels on {n} threads (mean {per_frame:.2f} s)"}
    gpu_ref = reference_gpu(frame)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_frame * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args.workload, frame, world),
            "cpu_baseline": info, "reference_gpu": gpu_ref,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_of(workload, frame, world=1):
    """The config object both arms print for a single-frame workload (the same keys and
    values in both, so that the two lines describe one workload)."""
    return {"workload": WORKLOADS[workload], "n_vox": frame.n_vox, "n_sv": frame.n_sv, "n_gauss": frame.n_gauss,
            "em_iterations": EM_ITERS, "l2": "inputs larger than L2 (16 B x n_vox)" if workload == "c2" else
            "inputs fit in L2", "ll_precision": "mixed", "ll_mode": "as_reference",
            "parallelism": f"replicas x{world}"}


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
    # the autotuner picks the kNN/E-step width on this frame (untimed; results do not depend on it)
    if args.knn_lanes:
        plan.set_knn_group(args.knn_lanes)
        plan.set_knn_fusion(bool(args.knn_fused))
        knn_lanes = args.knn_lanes
    else:
        knn_lanes = plan.autotune([df], [gm], [rnk], [ind], params, reps=3)
    knn_fused = plan.tuning()["knn_fused"]

    def step():
        gm.copy_(gm0, non_blocking=True)
        plan.run_device(df, gm, rnk, ind, params, stats=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    check = plan.run_device(df, gm.copy_(gm0), rnk, ind, params, stats=True)
    assert check["iterations"] == EM_ITERS, check
    got = {"gauss": gm.cpu().numpy().view(L.GAUSS_DTYPE).copy(), "rnk": rnk.cpu().numpy(), "ind": ind.cpu().numpy(),
           "ll": check["ll"]}

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
    value, voxel_iters, max_ms, total_vox = reduce_job(total_ms, N, args.steps, world, dev)

    # roofline of the dominant kernel, timed alone on this stream on the same workload: the
    # per-iteration voxel pass, or, when the autotuner made it run the next iteration's
    # kNN/E-step, that form.  Algorithmic bytes: 16 B per voxel (x, y, z, I); the kNN/E-step
    # adds 164 B per supervoxel (centroid, CSR bounds, 9 moments, neighbour list, candidates
    # and responsibilities out) and 104 B per Gaussian (E-step record, float centre).
    ms_llk = plan_time(plan, L.TGMM_KERNEL_LL_PASS_KNN, 20, stream)
    ms_ll = plan_time(plan, L.TGMM_KERNEL_LL_PASS, 20, stream)
    ms_mom = plan_time(plan, L.TGMM_KERNEL_MOMENTS, 10, stream)
    peak, peak_kind = measured_peaks()
    vox_bytes = 16.0 * N
    knn_bytes = 164.0 * S + 104.0 * K
    alone = {"kernel": "k_ll_pass<0, 0, 0> (the voxel pass alone)", "ms_per_launch": ms_ll,
             "algorithmic_bytes_per_launch": vox_bytes, "achieved": vox_bytes / (ms_ll * 1e-3) / 1e9,
             "frac": vox_bytes / (ms_ll * 1e-3) / 1e9 / peak}
    fused = {"kernel": f"k_ll_pass<0, {max(knn_lanes, 8)}, 0> (the voxel pass running the next iteration's kNN/E-step)",
             "ms_per_launch": ms_llk, "algorithmic_bytes_per_launch": vox_bytes + knn_bytes,
             "achieved": (vox_bytes + knn_bytes) / (ms_llk * 1e-3) / 1e9,
             "frac": (vox_bytes + knn_bytes) / (ms_llk * 1e-3) / 1e9 / peak}
    top, other = (fused, alone) if knn_fused else (alone, fused)
    traffic = committed_traffic(top["kernel"].split(" (")[0])
    roofline = {"bound": "hbm", "kernel": top["kernel"] + ", per iteration",
                "achieved": top["achieved"], "peak": peak, "unit": "GB/s", "frac": top["frac"],
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else
                "fallback 6650 GB/s", "algorithmic_bytes_per_launch": top["algorithmic_bytes_per_launch"],
                "ms_per_launch": top["ms_per_launch"],
                "traffic": (traffic["bytes_per_launch"] * N / traffic["n_vox"]) if traffic else None,
                "other_form": other,
                "moments_pass": {"ms_per_launch": ms_mom, "achieved": vox_bytes / (ms_mom * 1e-3) / 1e9,
                                 "frac": vox_bytes / (ms_mom * 1e-3) / 1e9 / peak}}

    # end to end through the C ABI with host buffers: H2D of the frame, Gaussians H2D/D2H
    # inside tgmm_em_run, D2H of rnk/ind, every step
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(frame, df, plan, params, dev, args, form="runs")
        e2e["compact_6_bytes"] = run_e2e(frame, df, plan, params, dev, args, form="compact")
        e2e["float_arrays"] = run_e2e(frame, df, plan, params, dev, args, form="float")

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = cpu_baseline(frame, single=True)
        parity = parity_vs_oracle(frame, got)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": config_of(args.workload, frame, world),
                "tuning": {"knn_lanes_per_supervoxel": knn_lanes, "knn_in_voxel_pass": knn_fused,
                           "knn_grid_searches_after_iteration_1": check["knn_searches"]},
                "voxel_iters_per_s": voxel_iters,
                "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
                "gpu_launches": kernels_per_call(knn_fused) * args.steps,
                "roofline": roofline, "clocks": clocks.summary(), "e2e": e2e, "cpu_baseline": cpu,
                "parity": parity}
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


def run_e2e(frame, df, plan, params, dev, args, form="runs"):
    """End to end through the C ABI with host buffers, every step: the frame's upload from
    page-locked memory, tgmm_em_run (its Gaussians up and down inside), rnk/ind down.  The
    upload of step i + 1 runs on a copy stream into the other of two buffers while step i's EM
    runs (the expansion of a compact form runs there too), so a step costs the slower of the
    two.  form "runs": the voxels cross as runs of
    consecutive linear indices (uint32 start, uint16 length, per supervoxel int32 run pointers)
    and uint16 raw values, about 3 bytes a voxel, and tgmm_frame_expand_runs rebuilds the float
    arrays on the device; "compact": 6 bytes a voxel (uint32 linear index, uint16 raw value)
    through tgmm_frame_expand; "float": the float arrays of the reference's layout (16 bytes a
    voxel)."""
    import ctypes as C
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    N, S, K = frame.n_vox, frame.n_sv, frame.n_gauss

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    compact = form != "float"
    if form == "runs":
        rp, rs, rl, raw, dims, off, den = frame.runs()
        host = {"run_ptr": pinned(rp), "run_start": pinned(rs.view(np.int32)), "run_len": pinned(rl.view(np.int16)),
                "raw": pinned(raw.view(np.int16))}
    elif form == "compact":
        lin, raw, dims, off, den = frame.compact()
        host = {"lin": pinned(lin.view(np.int32)), "raw": pinned(raw.view(np.int16))}
    else:
        host = {"query": pinned(frame.query), "img": pinned(frame.img)}
    host.update(centroids=pinned(frame.centroids), label_ptr=pinned(frame.label_ptr))
    bufs = [{k: torch.empty_like(v, device=dev) for k, v in host.items()} for _ in range(2)]
    if compact:  # the expanded float arrays, one pair per buffer
        for b in bufs:
            b["query"] = torch.empty_like(df.query)
            b["img"] = torch.empty_like(df.img)
    rnk_h = torch.empty(5 * S, dtype=torch.float32).pin_memory()
    ind_h = torch.empty(5 * S, dtype=torch.int32).pin_memory()
    rnk = torch.empty(5 * S, dtype=torch.float32, device=dev)
    ind = torch.empty(5 * S, dtype=torch.int32, device=dev)
    g0 = np.ascontiguousarray(frame.gauss.astype(L.GAUSS_DTYPE))
    comp = torch.cuda.current_stream(dev)
    cs = torch.cuda.Stream(dev)
    up = [torch.cuda.Event() for _ in range(2)]
    used = [torch.cuda.Event() for _ in range(2)]
    st = L.TgmmEmStats()
    lib = L.gmem()
    h2d = sum(int(v.numel() * v.element_size()) for v in host.values()) + 288 * K
    d2h = 288 * K + 8 * 5 * S

    def upload(i):
        """Step i's frame into buffer i % 2 on the copy stream, expanded there on the device."""
        b = bufs[i % 2]
        with torch.cuda.stream(cs):
            cs.wait_event(used[i % 2])  # the EM that read this buffer two steps ago is done
            for k, v in host.items():
                b[k].copy_(v, non_blocking=True)
            if form == "runs":
                E.expand_runs(b["run_ptr"], b["run_start"], b["run_len"], b["raw"], b["label_ptr"], dims, off, den,
                              b["query"], b["img"], stream=cs)
            elif form == "compact":
                E.expand_frame(b["lin"], b["raw"], dims, off, den, b["query"], b["img"], stream=cs)
            up[i % 2].record(cs)

    def run(n):
        gs = [torch.from_numpy(g0.view(np.uint8).copy()).pin_memory() for _ in range(n)]
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(comp)
        cs.wait_event(a)
        upload(0)
        t0 = time.perf_counter()
        for i in range(n):
            if i + 1 < n:
                upload(i + 1)
            b = bufs[i % 2]
            comp.wait_event(up[i % 2])
            f = E.DeviceFrame(b["query"], b["img"], b["centroids"], b["label_ptr"], K)
            cf = f.cframe()
            L.check(lib.tgmm_em_run(plan.h, C.byref(cf), gs[i].data_ptr(), rnk.data_ptr(), ind.data_ptr(), None,
                                    C.byref(params), C.byref(st), comp.cuda_stream), "tgmm_em_run")
            rnk_h.copy_(rnk, non_blocking=True)
            ind_h.copy_(ind, non_blocking=True)
            used[i % 2].record(comp)
        z.record(comp)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(z), time.perf_counter() - t0

    run(max(1, args.warmup))
    ms, wall = run(args.steps)
    return {"value": args.steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "wall_frames_per_s": args.steps / wall,
            "path": {"runs": "tgmm_frame_expand_runs + tgmm_em_run (C ABI): pinned voxel runs (uint32 start, uint16 "
                             "length, int32 pointer per supervoxel) and uint16 raw values (~3 B a voxel), centroids, "
                             "CSR and Gaussians up, rnk/ind and Gaussians down; uploads one step ahead on a copy stream",
                     "compact": "tgmm_frame_expand + tgmm_em_run (C ABI): pinned compact voxels (6 B), centroids, CSR "
                                "and Gaussians up, rnk/ind and Gaussians down; uploads one step ahead on a copy stream",
                     "float": "tgmm_em_run (C ABI): pinned float arrays (16 B a voxel, the reference's layout), "
                              "centroids, CSR and Gaussians up, rnk/ind and Gaussians down; uploads one step ahead on "
                              "a copy stream"}[form]}


# ---------------------------------------------------------------------------
# Batched and served forms (non-default workloads; one JSON line each)
# ---------------------------------------------------------------------------
def _pin(frame):
    """The frame as the served and plain forms upload it: its voxel runs (int32 pointer per
    supervoxel, uint32 start, uint16 length) and uint16 raw values, centroids and CSR copied
    once into page-locked memory (numpy views), and its first-frame Gaussians; the float
    arrays are not kept (a series of hundreds of 1-Gvoxel frames would not fit the host's
    memory in float form)."""
    import torch

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    rp, rs, rl, raw, dims, off, den = frame.runs()
    out = dict(centroids=pinned(frame.centroids), label_ptr=pinned(frame.label_ptr), run_ptr=pinned(rp),
               run_start=pinned(rs.view(np.int32)).view(np.uint32), run_len=pinned(rl.view(np.int16)).view(np.uint16),
               raw=pinned(raw.view(np.int16)).view(np.uint16),
               dims=dims, raw_offset=off, raw_denom=den, n_vox=frame.n_vox, n_sv=frame.n_sv, gauss=frame.gauss)
    return type("PinnedFrame", (), out)


def _lin_of(f):
    """A pinned frame's linear voxel indices, rebuilt on the host from its runs."""
    rl = f.run_len.astype(np.int64)
    pos = np.arange(int(rl.sum())) - np.repeat(np.cumsum(rl) - rl, rl)
    return np.repeat(f.run_start.astype(np.int64), rl) + pos


def run_batch64(args):
    """64 independent volumes (uneven sizes): one tgmm_em_run_batch call per step (one
    launch per EM phase for all volumes) against the same volumes one at a time through
    tgmm_em_run_device; inputs resident on the device, 20 iterations each."""
    import torch
    from tgmm_b200 import engine as E
    from tgmm_b200 import synth
    torch.cuda.set_device(0)
    specs = synth.batch_specs(64, seed=args.seed)
    frames = [synth.generate(sp, seed=args.seed + i) for i, sp in enumerate(specs)]
    prm = synth.em_params(iters=EM_ITERS, tol=-1.0)
    dfs = [E.to_device(f) for f in frames]
    gm0 = [E.gauss_to_device(f.gauss) for f in frames]
    gms = [g.clone() for g in gm0]
    rnks = [torch.empty(5 * f.n_sv, device="cuda") for f in frames]
    inds = [torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda") for f in frames]
    tv, ts, tg = sum(f.n_vox for f in frames), sum(f.n_sv for f in frames), sum(f.n_gauss for f in frames)
    batch_plan = E.Plan(tv, ts, tg, max_frames=len(frames))
    one_plan = E.Plan(max(f.n_vox for f in frames), max(f.n_sv for f in frames), max(f.n_gauss for f in frames))
    # tuned on the batch, and on its median volume for the one-at-a-time plan (untimed)
    lanes_b = batch_plan.autotune(dfs, gms, rnks, inds, prm, reps=2)
    fused_b = batch_plan.tuning()["knn_fused"]
    mid = sorted(range(len(frames)), key=lambda i: frames[i].n_vox)[len(frames) // 2]
    lanes_p = one_plan.autotune([dfs[mid]], [gms[mid]], [rnks[mid]], [inds[mid]], prm, reps=3)
    fused_p = one_plan.tuning()["knn_fused"]

    def batched():
        for g, g0 in zip(gms, gm0):
            g.copy_(g0)
        batch_plan.run_batch(dfs, gms, rnks, inds, prm, stats=False)

    def plain():
        for df, g, g0, r, i in zip(dfs, gms, gm0, rnks, inds):
            g.copy_(g0)
            one_plan.run_device(df, g, r, i, prm, stats=False)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    ms_b = timed(batched)
    out_b = [(r.cpu().numpy(), i.cpu().numpy()) for r, i in zip(rnks, inds)]
    ms_p = timed(plain)
    same = all(np.array_equal(rb, r.cpu().numpy()) and np.array_equal(ib, i.cpu().numpy())
               for (rb, ib), r, i in zip(out_b, rnks, inds))
    n = len(frames)
    line = {"metric": "EM frames/s, 64 uneven volumes batched", "value": n / (ms_b / 1e3), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "64 volumes, dims uniform in [128..512]x[128..512]x[64..128], one nucleus per "
                                   "~3000 voxels clipped to [100, 5000], 20 EM iterations",
                       "total_vox": tv, "total_sv": ts, "total_gauss": tg},
            "plain": {"value": n / (ms_p / 1e3), "ms_per_sweep": ms_p, "path": "tgmm_em_run_device, one at a time"},
            "batched_over_plain": ms_p / ms_b, "voxel_iters_per_s": tv * EM_ITERS / (ms_b / 1e3),
            "knn_lanes_per_supervoxel": {"batched": lanes_b, "plain": lanes_p},
            "knn_in_voxel_pass": {"batched": fused_b, "plain": fused_p},
            "rnk_ind_identical_to_alone": bool(same)}
    print(json.dumps(line), flush=True)


SERIES_SPECS = {
    "series": [((1024, 1024, 256), 5000)],
    "mixed": [((256, 256, 64), 300), ((512, 512, 128), 2000), ((1024, 1024, 256), 8000), ((2048, 1024, 512), 20000)],
}
SERIES_FRAMES = {"series": 200, "mixed": 100}  # frames per series of the served configurations
SERIES_RATE = {"series": 2.0, "mixed": 8.0}    # Poisson arrivals per second, all series together


def _series(args):
    """The time series of the workload, each frame kept only in its pinned run form."""
    from tgmm_b200 import synth
    nf = args.frames or SERIES_FRAMES[args.workload]
    out = []
    for i, (dims, n) in enumerate(SERIES_SPECS[args.workload]):
        spec = synth.VolumeSpec(dims=dims, n_nuclei=n, axis_min=4.0, axis_max=8.0)
        out.append([_pin(f) for f in synth.time_series_iter(spec, seed=args.seed + 17 * i, n_frames=nf,
                                                              divide_frac=0.01)])
    return out


def run_served(args):
    """Served time series: the server (tgmm_serve.h) against the plain form, both over the
    same pinned frames as voxel runs (about 3 bytes a voxel, expanded on the device), both returning
    rnk/ind and the posterior of every frame and carrying each lineage's posterior into its
    next frame's prior on the device.  Closed loop (every frame submitted at once) gives
    throughput; Poisson arrivals at the configured rate give per-frame latency."""
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    from tgmm_b200.serve import Server
    torch.cuda.set_device(0)
    t_gen = time.perf_counter()
    series = _series(args)
    t_gen = time.perf_counter() - t_gen
    from tgmm_b200 import synth
    prm = synth.em_params(iters=EM_ITERS, tol=1e-6)
    order = [(li, t) for t in range(len(series[0])) for li in range(len(series))]  # interleaved arrivals
    n_frames = len(order)
    rate = SERIES_RATE[args.workload]

    # plain form: one frame at a time
    K = [fr[0].gauss.shape[0] for fr in series]
    maxN = max(f.n_vox for fr in series for f in fr)
    maxS = max(f.n_sv for fr in series for f in fr)
    plan = E.Plan(maxN, maxS, max(K))
    maxR = max(f.run_start.shape[0] for fr in series for f in fr)
    rp_d = torch.empty(maxS + 1, dtype=torch.int32, device="cuda")
    rs_d = torch.empty(maxR, dtype=torch.int32, device="cuda")
    rl_d = torch.empty(maxR, dtype=torch.int16, device="cuda")
    raw_d = torch.empty(maxN, dtype=torch.int16, device="cuda")
    q = torch.empty(3 * maxN, device="cuda")
    im = torch.empty(maxN, device="cuda")
    ce = torch.empty(3 * maxS, device="cuda")
    lp = torch.empty(maxS + 1, dtype=torch.int64, device="cuda")
    rnk = torch.empty(5 * maxS, device="cuda")
    ind = torch.empty(5 * maxS, dtype=torch.int32, device="cuda")
    rnk_h = torch.empty(5 * maxS).pin_memory()
    ind_h = torch.empty(5 * maxS, dtype=torch.int32).pin_memory()

    def plain_sweep():
        gms = [E.gauss_to_device(fr[0].gauss) for fr in series]
        gm_h = [torch.empty(k * 288, dtype=torch.uint8).pin_memory() for k in K]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for li, t in order:
            f = series[li][t]
            N, S = f.n_vox, f.n_sv
            R = f.run_start.shape[0]
            rp_d[:S + 1].copy_(torch.from_numpy(f.run_ptr), non_blocking=True)
            rs_d[:R].copy_(torch.from_numpy(f.run_start.view(np.int32)), non_blocking=True)
            rl_d[:R].copy_(torch.from_numpy(f.run_len.view(np.int16)), non_blocking=True)
            raw_d[:N].copy_(torch.from_numpy(f.raw.view(np.int16)), non_blocking=True)
            ce[:3 * S].copy_(torch.from_numpy(f.centroids), non_blocking=True)
            lp[:S + 1].copy_(torch.from_numpy(f.label_ptr), non_blocking=True)
            E.expand_runs(rp_d[:S + 1], rs_d[:R], rl_d[:R], raw_d[:N], lp[:S + 1], f.dims, f.raw_offset, f.raw_denom,
                          q[:3 * N], im[:N])
            df = E.DeviceFrame(q[:3 * N], im[:N], ce[:3 * S], lp[:S + 1], K[li])
            plan.run_device(df, gms[li], rnk, ind, prm, stats=True)
            rnk_h[:5 * S].copy_(rnk[:5 * S], non_blocking=True)
            ind_h[:5 * S].copy_(ind[:5 * S], non_blocking=True)
            gm_h[li].copy_(gms[li].view(torch.uint8), non_blocking=True)
            E.update_priors(gms[li], K[li])
            torch.cuda.synchronize()
        return time.perf_counter() - t0

    qf_h = torch.empty(3 * maxN).pin_memory()
    imf_h = torch.empty(maxN).pin_memory()

    def float_frame(f):
        """The frame's float arrays in the reference's layout, rebuilt on the host from its
        voxel runs (the values the generator produced, bit for bit)."""
        X, Y, _ = f.dims
        lin = _lin_of(f)
        N = f.n_vox
        q = qf_h[:3 * N].numpy().reshape(3, N)
        q[0] = lin % X
        q[1] = (lin // X) % Y
        q[2] = lin // (X * Y)
        imf_h[:N].numpy()[:] = ((f.raw.astype(np.float64) - f.raw_offset) / f.raw_denom).astype(np.float32)

    def plain_float_sweep():
        """The plain form with the reference's float arrays (16 B a voxel) uploaded: per frame
        the same work as plain_sweep; the host-side rebuild of each frame's float arrays into
        the page-locked staging buffers happens between frames and is not timed."""
        gms = [E.gauss_to_device(fr[0].gauss) for fr in series]
        gm_h = [torch.empty(k * 288, dtype=torch.uint8).pin_memory() for k in K]
        torch.cuda.synchronize()
        total = 0.0
        for li, t in order:
            f = series[li][t]
            N, S = f.n_vox, f.n_sv
            float_frame(f)
            t0 = time.perf_counter()
            q[:3 * N].copy_(qf_h[:3 * N], non_blocking=True)
            im[:N].copy_(imf_h[:N], non_blocking=True)
            ce[:3 * S].copy_(torch.from_numpy(f.centroids), non_blocking=True)
            lp[:S + 1].copy_(torch.from_numpy(f.label_ptr), non_blocking=True)
            df = E.DeviceFrame(q[:3 * N], im[:N], ce[:3 * S], lp[:S + 1], K[li])
            plan.run_device(df, gms[li], rnk, ind, prm, stats=True)
            rnk_h[:5 * S].copy_(rnk[:5 * S], non_blocking=True)
            ind_h[:5 * S].copy_(ind[:5 * S], non_blocking=True)
            gm_h[li].copy_(gms[li].view(torch.uint8), non_blocking=True)
            E.update_priors(gms[li], K[li])
            torch.cuda.synchronize()
            total += time.perf_counter() - t0
        return total

    for _ in range(max(1, args.warmup)):
        plain_sweep()
    plain_s = min(plain_sweep() for _ in range(max(1, min(args.steps, 3))))
    plain_float_s = plain_float_sweep()

    # served form; outputs into page-locked buffers, as the plain form's
    srv = Server(params=prm, lanes=2, max_batch_frames=16, max_batch_vox=max(1 << 25, 2 * maxN))

    def pinned_out(S, K):
        return (torch.empty(5 * S).pin_memory().numpy(), torch.empty(5 * S, dtype=torch.int32).pin_memory().numpy(),
                torch.empty(K * 288, dtype=torch.uint8).pin_memory().numpy().view(L.GAUSS_DTYPE))
    # one output set per frame of a time step (a lineage's frames run in order, so a step's
    # outputs are free again once the next step of that lineage has started)
    outs = [[pinned_out(max(f.n_sv for f in fr), K[li]) for _ in range(2)] for li, fr in enumerate(series)]

    def served(arrival_rate=None, seed=0):
        ids = [srv.open_lineage(fr[0].gauss) for fr in series]
        rng = np.random.default_rng(seed)
        t0 = time.perf_counter()
        t_next = 0.0
        res = []
        for n, (li, t) in enumerate(order):
            if arrival_rate:
                t_next += rng.exponential(1.0 / arrival_rate)
                while time.perf_counter() - t0 < t_next:
                    res.extend(srv.poll(wait_ms=0))
                    time.sleep(0.0005)
            srv.submit(ids[li], series[li][t], tag=n, runs=True, out=outs[li][t % 2])
        res.extend(srv.drain())
        wall = time.perf_counter() - t0
        for i in ids:
            srv.close_lineage(i)
        bad = [r.status for r in res if r.status != L.TGMM_OK]
        return wall, res, bad

    for _ in range(max(1, args.warmup)):
        served()
    h2d0 = srv.stats()["h2d_bytes"]
    closed = [served() for _ in range(max(1, min(args.steps, 3)))]
    wall_c, res_c, bad_c = min(closed, key=lambda x: x[0])
    h2d_frame = (srv.stats()["h2d_bytes"] - h2d0) / len(closed) / n_frames
    wall_o, res_o, bad_o = served(arrival_rate=rate, seed=args.seed)
    lat = sorted(r.latency_ms for r in res_o)
    st = srv.stats()
    srv.close()
    pct = lambda a, p: float(np.percentile(a, p))
    line = {"metric": f"served EM frames/s ({args.workload} stream)", "value": n_frames / wall_c, "unit": UNIT,
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": [f"{d[0]}x{d[1]}x{d[2]}, {n} nuclei" for d, n in SERIES_SPECS[args.workload]],
                       "frames_per_series": len(series[0]), "frames": n_frames, "em": "max 20 iterations, tol 1e-6",
                       "n_vox_per_series": [[min(f.n_vox for f in fr), max(f.n_vox for f in fr)] for fr in series],
                       "lanes": 2, "upload": "voxel runs and raw values (~3 B a voxel), expanded on the device, "
                                             "both forms",
                       "generation_s": round(t_gen, 1)},
            "plain": {"value": n_frames / plain_s, "unit": UNIT,
                      "path": "one frame at a time: pinned run upload, tgmm_frame_expand_runs, tgmm_em_run_device, "
                              "download, prior update"},
            "plain_float_arrays": {"value": n_frames / plain_float_s, "unit": UNIT,
                                   "path": "one frame at a time as above, the frame uploaded as the reference's "
                                           "float arrays (16 B a voxel) instead of voxel runs; the host-side "
                                           "rebuild of those arrays between frames is not timed"},
            "served_over_plain": (n_frames / wall_c) / (n_frames / plain_s),
            "served_over_plain_float_arrays": (n_frames / wall_c) / (n_frames / plain_float_s),
            "h2d_bytes_per_frame": h2d_frame,
            "latency_ms": {"arrivals_per_s": rate, "frames": len(lat), "p50": pct(lat, 50), "p99": pct(lat, 99),
                           "max": lat[-1], "wall_s": wall_o},
            "closed_loop_latency_ms": {"p50": pct([r.latency_ms for r in res_c], 50),
                                       "p99": pct([r.latency_ms for r in res_c], 99)},
            "mean_batch_frames": st["frames_in_batches"] / max(1, st["batches"]),
            "mean_em_iterations_per_series": [float(np.mean([r.stats["iterations"] for r in res_c
                                                             if order[r.tag][0] == li]))
                                              for li in range(len(series))],
            "hbm_peak_bytes": st["hbm_peak"], "errors": bad_c + bad_o}
    print(json.dumps(line), flush=True)


FB_STAGES = ["clear+init", "k_fb_scan", "k_fb_ptr", "k_fb_group", "k_fb_trim", "k_fb_order", "k_fb_csr", "k_fb_emit"]


def fb_volume(spec, seed, device):
    """A synthetic frame's supervoxels scattered into full volumes on the device: the raw
    image (background 100-129, the frame's foreground values) and the label volume (its
    supervoxels, 1-based).  Returns (raw int16, label int32, n_labels, labelled voxels,
    summed bounding-box voxels, lists): lists holds the same segmentation as per-supervoxel
    pixel lists on the device (lin int32 bits of uint32 indices, val int16 bits of the raw
    values, ptr int64), the form tgmm_frame_build_lists reads."""
    import torch
    from tgmm_b200 import synth
    fr = synth.make_frame(spec, synth.random_nuclei(spec, seed), seed)
    synth.release(fr)
    X, Y, Z = spec.dims
    nvol, N, S = X * Y * Z, fr.n_vox, fr.n_sv
    q = fr.query.reshape(3, N)
    lp = fr.label_ptr
    lo = np.minimum.reduceat(q, lp[:-1], axis=1) if N else np.zeros((3, S))
    hi = np.maximum.reduceat(q, lp[:-1], axis=1) if N else np.zeros((3, S))
    box = int(np.prod(hi - lo + 1, axis=0).sum())
    qd = torch.from_numpy(fr.query).to(device).view(3, N).long()
    lin = qd[0] + X * (qd[1] + Y * qd[2])
    del qd
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    raw = torch.randint(100, 130, (nvol,), device=device, generator=g, dtype=torch.int32)
    raw[lin] = torch.from_numpy(fr.raw.astype(np.int32)).to(device)
    raw = raw.to(torch.int16)
    lab = torch.zeros(nvol, dtype=torch.int32, device=device)
    lab[lin] = torch.repeat_interleave(torch.arange(1, S + 1, device=device, dtype=torch.int32),
                                       torch.from_numpy(np.diff(lp)).to(device))
    lists = {"lin": lin.to(torch.int32), "val": raw[lin].clone(),
             "ptr": torch.from_numpy(np.ascontiguousarray(lp, np.int64)).to(device)}
    return raw, lab, S, N, box, lists


def run_frames(args):
    """Frame preparation (tgmm_frame_build) of one volume per rank: value = volumes per second
    over all ranks, with the raw and label volumes resident; e2e adds their upload from pinned
    host memory every step."""
    import torch
    import torch.distributed as dist
    from tgmm_b200 import engine as E
    from tgmm_b200 import synth
    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    spec = fb_spec(args)
    raw, lab, S, Nfg, box, lists = fb_volume(spec, args.seed + rank, dev)
    X, Y, Z = spec.dims
    nvol = X * Y * Z
    b = E.FrameBuilder((X, Y, Z), S, device=dev, max_vox=Nfg)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        b.build(raw, lab, read_thr=False)
    stages = []
    for _ in range(3):
        ms = []
        b.build(raw, lab, stage_ms=ms, read_thr=False)
        stages.append(ms)
    stage = np.mean(np.array(stages), axis=0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            f, _ = b.build(raw, lab, read_thr=False)
        e1.record(stream)
        torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * args.steps / (max_ms / 1e3)
    e2e = None
    if not args.no_e2e:
        raw_h, lab_h = raw.cpu().pin_memory(), lab.cpu().pin_memory()
        for _ in range(2):
            raw.copy_(raw_h, non_blocking=True)
            lab.copy_(lab_h, non_blocking=True)
            b.build(raw, lab, read_thr=False)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            raw.copy_(raw_h, non_blocking=True)
            lab.copy_(lab_h, non_blocking=True)
            b.build(raw, lab, read_thr=False)
        e1.record(stream)
        torch.cuda.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": world * args.steps / (float(te.item()) / 1e3), "unit": "volumes/s",
               "h2d_bytes_per_step": 6 * nvol, "d2h_bytes_per_step": 64,
               "path": "pinned raw + label upload, then tgmm_frame_build (reads its sizes back)"}
    # the same segmentation as per-supervoxel pixel lists (the tracking program's form): no
    # volume on the device, so no scan; outputs compared with the volume form's
    ql, il = f.query.clone(), f.img.clone()
    lin_d, val_d, ptr_d = lists["lin"], lists["val"], lists["ptr"]
    for _ in range(args.warmup):
        b.build_lists(lin_d, val_d, ptr_d, read_thr=False)
    lstages = []
    for _ in range(3):
        ms = []
        fl, _ = b.build_lists(lin_d, val_d, ptr_d, stage_ms=ms, read_thr=False)
        lstages.append(ms)
    same_lists = bool(fl.n_vox == f.n_vox and torch.equal(fl.query, ql) and torch.equal(fl.img, il))
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        b.build_lists(lin_d, val_d, ptr_d, read_thr=False)
    e1.record(stream)
    torch.cuda.synchronize()
    tl = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tl, op=dist.ReduceOp.MAX)
    lists_line = {"value": world * args.steps / (float(tl.item()) / 1e3), "unit": "volumes/s",
                  "stage_ms": dict(zip(["clear+init", "k_fbl_boxes", "(no CSR step)", "(no grouping step)", "k_fb_trim",
                                        "k_fb_order", "k_fb_csr", "k_fb_emit"],
                                       [round(float(x), 4) for x in np.mean(np.array(lstages), axis=0)])),
                  "same_outputs_as_volume_form": same_lists,
                  "path": "tgmm_frame_build_lists: per-supervoxel pixel lists (uint32 linear indices, uint16 raw "
                          "values, int64 CSR) resident"}
    if not args.no_e2e:
        # every step uploads its volume's lists from pinned memory into one of two buffers on a
        # copy stream, one step ahead of the build that reads them
        host = {k: v.cpu().pin_memory() for k, v in lists.items()}
        bufs = [{k: torch.empty_like(v) for k, v in lists.items()} for _ in range(2)]
        cs = torch.cuda.Stream(dev)
        up = [torch.cuda.Event() for _ in range(2)]
        used = [torch.cuda.Event() for _ in range(2)]

        def upload(i):
            with torch.cuda.stream(cs):
                cs.wait_event(used[i % 2])
                for k in host:
                    bufs[i % 2][k].copy_(host[k], non_blocking=True)
                up[i % 2].record(cs)

        def run(n):
            torch.cuda.synchronize()
            e0.record(stream)
            cs.wait_event(e0)
            upload(0)
            for i in range(n):
                if i + 1 < n:
                    upload(i + 1)
                stream.wait_event(up[i % 2])
                bb = bufs[i % 2]
                b.build_lists(bb["lin"], bb["val"], bb["ptr"], read_thr=False)
                used[i % 2].record(stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        run(2)
        te = torch.tensor([run(args.steps)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        lists_line["e2e"] = {"value": world * args.steps / (float(te.item()) / 1e3), "unit": "volumes/s",
                             "h2d_bytes_per_step": sum(int(v.numel() * v.element_size()) for v in host.values()),
                             "d2h_bytes_per_step": 64,
                             "path": "pinned pixel-list upload on a copy stream one step ahead, then "
                                     "tgmm_frame_build_lists (reads its sizes back)"}
    # roofline of the dominant step, from the events between the steps
    algo = {"k_fb_scan": 4 * nvol, "k_fb_group": 4 * box + 8 * Nfg,
            "k_fb_emit": 6 * Nfg + 16 * f.n_vox}
    top = int(np.argmax(stage))
    name = FB_STAGES[top]
    peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    if name in algo:
        ach = algo[name] / (stage[top] * 1e-3) / 1e9
        traffic = None
        try:  # the committed ncu capture of the scan on a smaller volume, scaled by its voxels
            with open(os.path.join(ROOT, "profiles", "frame_scan_traffic.json")) as fh:
                tr = json.load(fh)
            if name == tr["kernel"]:
                traffic = (tr["dram_bytes_read_per_launch"] + tr["dram_bytes_write_per_launch"]) / tr["n_voxels"] * nvol
        except Exception:
            pass
        roof = {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": traffic, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "algorithmic_bytes": algo[name]}
    else:
        roof = {"bound": "latency", "kernel": name, "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                "traffic": None}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        raw_n = raw.cpu().numpy().view(np.uint16).reshape(Z, Y, X)
        lab_n = lab.cpu().numpy().view(np.uint32).reshape(Z, Y, X)
        if O.ref_f1_available():
            lists = O.supervoxel_lists(lab_n, S)
            t0 = time.perf_counter()
            rc, o = O.ref_frame_build(raw_n, lab_n, S, max_vox=Nfg, lists=lists)
            dt = time.perf_counter() - t0
            kind, what = "reference", ("the tracking program's host build loop with the reference's own "
                                       "trimSupervoxel, weightedGaussianStatistics and erase compiled from its "
                                       "sources, one thread")
        else:
            t0 = time.perf_counter()
            rc, o = O.frame_build(raw_n, lab_n, S, max_vox=Nfg)
            dt = time.perf_counter() - t0
            kind, what = "port", "the oracle's single-thread C restatement of the reference's host build"
        cpu = {"value": 1.0 / dt, "unit": "volumes/s", "cores": 1, "kind": kind, "cpu_model": cpu_model(),
               "sample": f"the whole volume once through {what} ({dt:.2f} s)",
               "same_outputs": bool(rc == 0 and o["n_vox"] == f.n_vox and
                                    np.array_equal(o["img"], f.img.cpu().numpy()) and
                                    np.array_equal(o["query"], f.query.cpu().numpy()))}
    if rank == 0:
        line = {"metric": "frame preparations/s", "value": value, "unit": "volumes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16/u32 -> f32",
                "data": "synthetic (seeded nuclei volume; labels = its supervoxels)",
                "config": {"workload": f"frame preparation of a {X}x{Y}x{Z} uint16 volume with {S} labelled "
                                       f"supervoxels ({Nfg} labelled voxels): trim, erase, centroids, "
                                       f"background, [0,1] rescale, SoA/CSR",
                           "n_vox_out": f.n_vox, "n_sv_out": f.n_sv, "l2": "inputs larger than L2"},
                "stage_ms": dict(zip(FB_STAGES, [round(float(x), 4) for x in stage])),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(),
                "gpu_launches": 8 * args.steps, "pixel_lists": lists_line}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch64":
        run_batch64(args)
    elif args.workload in ("series", "mixed"):
        run_served(args)
    elif args.workload == "frames":
        run_frames(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
