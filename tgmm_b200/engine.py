"""Engine wrapper: device buffers (torch) + the C ABI of libtgmm_gmem.so.

PyTorch only provides device memory and streams here; every kernel is the engine's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


@dataclass
class DeviceFrame:
    query: torch.Tensor      # (3N,) float32
    img: torch.Tensor        # (N,) float32
    centroids: torch.Tensor  # (3S,) float32
    label_ptr: torch.Tensor  # (S+1,) int64
    n_gauss: int

    @property
    def n_vox(self):
        return int(self.img.numel())

    @property
    def n_sv(self):
        return int(self.label_ptr.numel() - 1)

    def cframe(self) -> L.TgmmFrame:
        f = L.TgmmFrame()
        f.query, f.img = self.query.data_ptr(), self.img.data_ptr()
        f.centroids, f.label_ptr = self.centroids.data_ptr(), self.label_ptr.data_ptr()
        f.n_vox, f.n_sv, f.n_gauss = self.n_vox, self.n_sv, self.n_gauss
        return f


def to_device(frame, device="cuda", pin=False, n_gauss: int | None = None) -> DeviceFrame:
    """Copy a synth.Frame (host arrays) to the device.  n_gauss: the Gaussians the frame
    runs with (default: the frame's own first-frame Gaussians)."""
    def t(a):
        x = torch.from_numpy(np.ascontiguousarray(a))
        if pin:
            x = x.pin_memory()
        return x.to(device, non_blocking=pin)
    return DeviceFrame(t(frame.query), t(frame.img), t(frame.centroids), t(frame.label_ptr),
                       frame.n_gauss if n_gauss is None else n_gauss)


def gauss_to_device(g: np.ndarray, device="cuda") -> torch.Tensor:
    return torch.from_numpy(L.records(g).view(np.uint8)).to(device)


def gauss_from_device(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(L.GAUSS_DTYPE).copy()


def stats_dict(st: L.TgmmEmStats) -> dict:
    return dict(iterations=st.iterations, converged=st.converged, ll=st.ll, ll_true=st.ll_true,
                ll_as_reference=st.ll_as_reference, total_alpha=st.total_alpha, n_dead=st.n_dead,
                device_flags=st.device_flags, knn_searches=st.knn_searches)


class Plan:
    """All device workspace of the EM for batches up to the given capacity."""

    def __init__(self, max_vox: int, max_sv: int, max_gauss: int, max_frames: int = 1, device: int = 0):
        self.lib = L.gmem()
        d = L.TgmmPlanDesc()
        d.max_vox, d.max_sv, d.max_gauss, d.max_frames, d.device = max_vox, max_sv, max(max_gauss, 5), max_frames, device
        self.desc = d
        h = C.c_void_p()
        L.check(self.lib.tgmm_plan_create(C.byref(d), C.byref(h)), "tgmm_plan_create")
        self.h = h

    @staticmethod
    def bytes_for(max_vox, max_sv, max_gauss, max_frames=1) -> int:
        d = L.TgmmPlanDesc()
        d.max_vox, d.max_sv, d.max_gauss, d.max_frames, d.device = max_vox, max_sv, max(max_gauss, 5), max_frames, 0
        return int(L.gmem().tgmm_plan_bytes(C.byref(d)))

    def close(self):
        if self.h:
            self.lib.tgmm_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- single frame, Gaussians on the host (the reference's ownership model) --
    def run_host(self, df: DeviceFrame, gauss: np.ndarray, params: L.TgmmEmParams, stream=None, want_ind_tr=False):
        g = L.records(gauss)
        S = df.n_sv
        rnk = torch.empty(5 * S, dtype=torch.float32, device=df.img.device)
        ind = torch.empty(5 * S, dtype=torch.int32, device=df.img.device)
        ind_tr = torch.empty(5 * S, dtype=torch.int32, device=df.img.device) if want_ind_tr else None
        st = L.TgmmEmStats()
        cf = df.cframe()
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        rc = self.lib.tgmm_em_run(self.h, C.byref(cf), g.ctypes.data, rnk.data_ptr(), ind.data_ptr(),
                                  ind_tr.data_ptr() if ind_tr is not None else None, C.byref(params), C.byref(st), s)
        L.check(rc, "tgmm_em_run")
        out = dict(gauss=g, rnk=rnk.cpu().numpy(), ind=ind.cpu().numpy(), **stats_dict(st))
        if ind_tr is not None:
            out["ind_tr"] = ind_tr.cpu().numpy()
        return out

    # -- device-resident form --
    def run_device(self, df: DeviceFrame, gm_dev: torch.Tensor, rnk: torch.Tensor, ind: torch.Tensor,
                   params: L.TgmmEmParams, stats: bool = True, stream=None):
        st = L.TgmmEmStats() if stats else None
        cf = df.cframe()
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        rc = self.lib.tgmm_em_run_device(self.h, C.byref(cf), gm_dev.data_ptr(), rnk.data_ptr(), ind.data_ptr(),
                                         C.byref(params), C.byref(st) if st is not None else None, s)
        L.check(rc, "tgmm_em_run_device")
        return stats_dict(st) if st is not None else None

    def run_batch(self, frames, gms, rnks, inds, params: L.TgmmEmParams, stats: bool = True, stream=None):
        n = len(frames)
        cfs = (L.TgmmFrame * n)(*[f.cframe() for f in frames])
        gp = (C.c_void_p * n)(*[g.data_ptr() for g in gms])
        rp = (C.c_void_p * n)(*[r.data_ptr() for r in rnks])
        ip = (C.c_void_p * n)(*[i.data_ptr() for i in inds])
        st = (L.TgmmEmStats * n)() if stats else None
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        rc = self.lib.tgmm_em_run_batch(self.h, n, cfs, gp, rp, ip, C.byref(params), st, s)
        L.check(rc, "tgmm_em_run_batch")
        return [stats_dict(x) for x in st] if st is not None else None


    def set_stage_wait(self, ns: int):
        """Wait limit of the voxel passes' tile copies (default 1 s)."""
        L.check(self.lib.tgmm_plan_set_stage_wait(self.h, int(ns)), "tgmm_plan_set_stage_wait")

    def run_host_status(self, df: DeviceFrame, gauss: np.ndarray, params: L.TgmmEmParams):
        """tgmm_em_run returning (status, stats) instead of raising on a non-zero status."""
        g = L.records(gauss)
        S = df.n_sv
        rnk = torch.empty(5 * S, dtype=torch.float32, device=df.img.device)
        ind = torch.empty(5 * S, dtype=torch.int32, device=df.img.device)
        st = L.TgmmEmStats()
        cf = df.cframe()
        rc = self.lib.tgmm_em_run(self.h, C.byref(cf), g.ctypes.data, rnk.data_ptr(), ind.data_ptr(), None,
                                  C.byref(params), C.byref(st), torch.cuda.current_stream().cuda_stream)
        return rc, stats_dict(st)

    def set_knn_group(self, lanes: int):
        L.check(self.lib.tgmm_plan_set_knn_group(self.h, lanes), "tgmm_plan_set_knn_group")

    def set_knn_fusion(self, on: bool):
        L.check(self.lib.tgmm_plan_set_knn_fusion(self.h, 1 if on else 0), "tgmm_plan_set_knn_fusion")

    def tuning(self) -> dict:
        """The kNN/E-step width and whether the voxel pass runs it (autotuned or set)."""
        lanes, fused = C.c_int32(), C.c_int32()
        L.check(self.lib.tgmm_plan_tuning(self.h, C.byref(lanes), C.byref(fused)), "tgmm_plan_tuning")
        return {"knn_lanes": lanes.value, "knn_fused": bool(fused.value)}

    def autotune(self, frames, gms, rnks, inds, params: L.TgmmEmParams, reps: int = 3, stream=None) -> int:
        """Runs the batch's EM call at every kNN/E-step width and arrangement and keeps the
        fastest pair (the Gaussians in gms are only read); returns the width (tuning() gives
        both)."""
        n = len(frames)
        cfs = (L.TgmmFrame * n)(*[f.cframe() for f in frames])
        gp = (C.c_void_p * n)(*[g.data_ptr() for g in gms])
        rp = (C.c_void_p * n)(*[r.data_ptr() for r in rnks])
        ip = (C.c_void_p * n)(*[i.data_ptr() for i in inds])
        out = C.c_int32()
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        L.check(self.lib.tgmm_plan_autotune(self.h, n, cfs, gp, rp, ip, C.byref(params), reps, C.byref(out), s),
                "tgmm_plan_autotune")
        return out.value


def knn(query: torch.Tensor, ref_xyz: torch.Tensor, scale=(1.0, 1.0, 2.0), stream=None) -> torch.Tensor:
    """Exact 5-NN (scaled squared distance, ties to the lower index); ind[j*nq + q]."""
    nq = query.numel() // 3
    ind = torch.empty(5 * nq, dtype=torch.int32, device=query.device)
    sc = (C.c_float * 3)(*scale)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.gmem().tgmm_knn(query.data_ptr(), nq, ref_xyz.data_ptr(), ref_xyz.numel() // 3, sc, ind.data_ptr(), s),
            "tgmm_knn")
    return ind


def expand_frame(lin: torch.Tensor, raw: torch.Tensor, dims, raw_offset: float, raw_denom: float,
                 query: torch.Tensor, img: torch.Tensor, stream=None):
    """tgmm_frame_expand: compact voxels (uint32 linear index, uint16 raw value; any 4- and
    2-byte dtypes) into the float query (3*n) and img (n) arrays on the device."""
    n = lin.numel()
    d = (C.c_int32 * 3)(*[int(x) for x in dims])
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.gmem().tgmm_frame_expand(lin.data_ptr(), raw.data_ptr(), n, d, float(raw_offset), float(raw_denom),
                                       query.data_ptr(), img.data_ptr(), s), "tgmm_frame_expand")


def expand_runs(run_ptr: torch.Tensor, run_start: torch.Tensor, run_len: torch.Tensor, raw: torch.Tensor,
                label_ptr: torch.Tensor, dims, raw_offset: float, raw_denom: float, query: torch.Tensor,
                img: torch.Tensor, stream=None):
    """tgmm_frame_expand_runs: runs (int32 run_ptr, 4-byte run_start, 2-byte run_len) and raw
    values (2-byte) over the CSR label_ptr into the float query (3*n) and img (n) arrays."""
    d = (C.c_int32 * 3)(*[int(x) for x in dims])
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.gmem().tgmm_frame_expand_runs(run_ptr.data_ptr(), run_start.data_ptr(), run_len.data_ptr(),
                                            raw.data_ptr(), label_ptr.data_ptr(), label_ptr.numel() - 1,
                                            run_start.numel(), raw.numel(), d, float(raw_offset), float(raw_denom),
                                            query.data_ptr(), img.data_ptr(), s), "tgmm_frame_expand_runs")


def local_likelihood(df: DeviceFrame, ind: torch.Tensor, gm_dev: torch.Tensor, lists, stream=None) -> np.ndarray:
    """tgmm_local_likelihood: one FP64 value per supervoxel list (host lists of supervoxel
    indices) under the Gaussians gm_dev (device records) with each supervoxel's candidates
    ind (device, slot-major 5*n_sv)."""
    ptr = np.zeros(len(lists) + 1, np.int32)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    idx = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in lists]) if ptr[-1] else
                               np.zeros(1, np.int32))
    out = np.zeros(len(lists), np.float64)
    cf = df.cframe()
    n_gauss = gm_dev.numel() // 288
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.gmem().tgmm_local_likelihood(C.byref(cf), ind.data_ptr(), gm_dev.data_ptr(), n_gauss, ptr.ctypes.data,
                                           idx.ctypes.data, len(lists), out.ctypes.data, s), "tgmm_local_likelihood")
    return out


def update_priors(gm_dev: torch.Tensor, n: int, beta_pct=0.01, nu_pct=1.0, alpha_pct=0.8, alpha_total=-1.0,
                  compute_alpha_total=True, stream=None):
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.gmem().tgmm_update_priors(gm_dev.data_ptr(), n, beta_pct, nu_pct, alpha_pct, alpha_total,
                                        1 if compute_alpha_total else 0, s), "tgmm_update_priors")


class FrameBuilder:
    """Frame preparation on the device (tgmm_frame_build) for volumes of one size: the raw
    16-bit image and the segmentation's label volume in, the EM's input arrays out.  The
    workspace and the output buffers are allocated once, for at most max_vox kept voxels
    (default: every voxel) and no supervoxel erased."""

    def __init__(self, dims, n_labels, device="cuda", max_nuclei_size=3000, max_percentile=0.4, conn3d=6,
                 min_nuclei_size=50, max_vox=None):
        self.lib = L.gmem()
        self.dims = (C.c_int32 * 3)(*dims)
        self.n_labels = int(n_labels)
        self.params = L.TgmmFrameBuildParams(max_nuclei_size, max_percentile, conn3d, min_nuclei_size)
        nbytes = self.lib.tgmm_frame_build_bytes(self.dims, self.n_labels)
        if nbytes < 0:
            raise ValueError("tgmm_frame_build_bytes: bad dimensions or label count")
        nvol = int(dims[0]) * int(dims[1]) * int(dims[2])
        self.nvol = nvol
        self.max_vox = nvol if max_vox is None else int(max_vox)
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.query = torch.empty(3 * self.max_vox, dtype=torch.float32, device=device)
        self.img = torch.empty(self.max_vox, dtype=torch.float32, device=device)
        self.cent = torch.empty(3 * self.n_labels, dtype=torch.float32, device=device)
        self.lptr = torch.empty(self.n_labels + 1, dtype=torch.int64, device=device)
        self.thr = torch.empty(self.n_labels, dtype=torch.int16, device=device)  # uint16 bits

    def build(self, raw: torch.Tensor, label: torch.Tensor, n_gauss: int = 0, stream=None, stage_ms=None,
              read_thr=True):
        """raw: uint16 bits (any 2-byte dtype), label: 4-byte labels (1..n_labels, 0 none), both
        X*Y*Z with x fastest.  Returns (DeviceFrame, thresholds as uint16 numpy or None).
        stage_ms: a list that receives each step's milliseconds (the timed form)."""
        if raw.numel() != self.nvol or label.numel() != self.nvol or raw.element_size() != 2 or \
                label.element_size() != 4:
            raise ValueError("raw must hold X*Y*Z 16-bit values and label X*Y*Z 32-bit labels")
        n_vox, n_sv = C.c_int64(0), C.c_int32(0)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        args = (raw.data_ptr(), label.data_ptr(), self.dims, self.n_labels, C.byref(self.params),
                self.workspace.data_ptr(), self.workspace.numel(), self.query.data_ptr(), self.img.data_ptr(),
                self.cent.data_ptr(), self.lptr.data_ptr(), self.thr.data_ptr(), self.max_vox, self.n_labels,
                C.byref(n_vox), C.byref(n_sv), s)
        if stage_ms is None:
            L.check(self.lib.tgmm_frame_build(*args), "tgmm_frame_build")
        else:
            ms = (C.c_float * L.TGMM_FRAME_BUILD_STAGES)()
            L.check(self.lib.tgmm_frame_build_timed(*args, ms), "tgmm_frame_build_timed")
            stage_ms[:] = list(ms)
        N, S = n_vox.value, n_sv.value
        f = DeviceFrame(self.query[:3 * N], self.img[:N], self.cent[:3 * S], self.lptr[:S + 1], n_gauss)
        return f, (self.thr[:S].cpu().numpy().view(np.uint16).copy() if read_thr else None)

    def build_lists(self, lin: torch.Tensor, val: torch.Tensor, lists_ptr: torch.Tensor, n_gauss: int = 0,
                    stream=None, stage_ms=None, read_thr=True):
        """tgmm_frame_build_lists: the segmentation as per-supervoxel pixel lists on the device
        -- lin (4-byte linear indices, ascending within each list), val (their 2-byte raw
        values), lists_ptr (int64, n_labels + 1) -- instead of volumes.  The same outputs as
        build().  The list workspace is allocated on first use for the largest list seen."""
        n_list = int(lin.numel())
        if val.numel() != n_list or val.element_size() != 2 or lin.element_size() != 4 or \
                lists_ptr.numel() != self.n_labels + 1 or lists_ptr.dtype != torch.int64:
            raise ValueError("lin and val need one entry per listed voxel, lists_ptr n_labels + 1 int64")
        nbytes = self.lib.tgmm_frame_build_lists_bytes(self.dims, self.n_labels, n_list)
        if nbytes < 0:
            raise ValueError("tgmm_frame_build_lists_bytes: bad sizes")
        if getattr(self, "list_ws", None) is None or self.list_ws.numel() < nbytes:
            self.list_ws = torch.empty(nbytes, dtype=torch.uint8, device=self.query.device)
        n_vox, n_sv = C.c_int64(0), C.c_int32(0)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        ms = (C.c_float * L.TGMM_FRAME_BUILD_STAGES)() if stage_ms is not None else None
        L.check(self.lib.tgmm_frame_build_lists(lin.data_ptr(), val.data_ptr(), lists_ptr.data_ptr(), n_list,
                                                self.dims, self.n_labels, C.byref(self.params),
                                                self.list_ws.data_ptr(), self.list_ws.numel(), self.query.data_ptr(),
                                                self.img.data_ptr(), self.cent.data_ptr(), self.lptr.data_ptr(),
                                                self.thr.data_ptr(), self.max_vox, self.n_labels, C.byref(n_vox),
                                                C.byref(n_sv), s, ms), "tgmm_frame_build_lists")
        if stage_ms is not None:
            stage_ms[:] = list(ms)
        N, S = n_vox.value, n_sv.value
        f = DeviceFrame(self.query[:3 * N], self.img[:N], self.cent[:3 * S], self.lptr[:S + 1], n_gauss)
        return f, (self.thr[:S].cpu().numpy().view(np.uint16).copy() if read_thr else None)
