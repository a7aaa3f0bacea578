"""Python face of the served form (include/tgmm_serve.h): lineages whose Gaussians stay on
the device, frames submitted from host memory, results polled back.

    srv = Server(params=synth.em_params(iters=20, tol=1e-6), lanes=2)
    lin = srv.open_lineage(first_frame.gauss)
    srv.submit(lin, frame, tag=0)              # host arrays of one time point
    for r in srv.poll(wait_ms=-1): ...          # ServeResult(tag, status, stats, rnk, ind, gauss, ...)

The server keeps a reference to every submitted frame's arrays (and their outputs) until
its result is polled, as the C API requires.  Frames of one lineage run in submission
order; frames of different lineages are batched together.

Multi-GPU: lineages are independent, so one server per GPU and a static assignment of
lineages to ranks (`lineage_shard`) covers N GPUs with no data exchange.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class ServeResult:
    tag: int
    lineage: int
    status: int
    stats: dict
    submit_ms: float
    start_ms: float
    done_ms: float
    batch_id: int
    batch_frames: int
    rnk: np.ndarray | None = None
    ind: np.ndarray | None = None
    gauss: np.ndarray | None = None

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


@dataclass
class _Pending:
    keep: list = field(default_factory=list)
    rnk: np.ndarray | None = None
    ind: np.ndarray | None = None
    gauss: np.ndarray | None = None


def _stats(st: L.TgmmEmStats) -> dict:
    return dict(iterations=st.iterations, converged=st.converged, ll=st.ll, ll_true=st.ll_true,
                ll_as_reference=st.ll_as_reference, total_alpha=st.total_alpha, n_dead=st.n_dead,
                device_flags=st.device_flags, knn_searches=st.knn_searches)


def lineage_shard(n_lineages: int, rank: int, world: int) -> list[int]:
    """Lineages of `rank` among `world` servers: a static round-robin split (every lineage
    on exactly one rank, sizes within one of each other)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, n_lineages, world))


class Server:
    def __init__(self, params: L.TgmmEmParams | None = None, device: int = 0, lanes: int = 2,
                 hbm_budget: int = 0, max_batch_frames: int = 64, max_batch_vox: int = 1 << 25,
                 max_batch_sv: int = 1 << 17, max_batch_gauss: int = 1 << 17, beta_pct: float = 0.01,
                 nu_pct: float = 1.0, alpha_pct: float = 0.8):
        lib = L.gmem()
        d = L.TgmmServerDesc()
        lib.tgmm_server_default_desc(C.byref(d))
        d.device, d.lanes, d.hbm_budget = device, lanes, hbm_budget
        d.max_batch_frames, d.max_batch_vox = max_batch_frames, max_batch_vox
        d.max_batch_sv, d.max_batch_gauss = max_batch_sv, max_batch_gauss
        if params is not None:
            d.params = params
        d.beta_pct, d.nu_pct, d.alpha_pct = beta_pct, nu_pct, alpha_pct
        self.desc = d
        h = C.c_void_p()
        L.check(lib.tgmm_server_create(C.byref(d), C.byref(h)), "tgmm_server_create")
        self.h = h
        self._pending: dict[int, _Pending] = {}
        self._n_gauss: dict[int, int] = {}

    def close(self):
        if self.h:
            L.check(L.gmem().tgmm_server_destroy(self.h), "tgmm_server_destroy")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open_lineage(self, gauss: np.ndarray) -> int:
        g = np.ascontiguousarray(gauss)
        if g.dtype.itemsize != 288:
            raise ValueError("Gaussian records must be the 288-byte GaussianMixtureModelCUDA layout")
        lid = C.c_int32()
        L.check(L.gmem().tgmm_server_open_lineage(self.h, g.ctypes.data, g.shape[0], C.byref(lid)),
                "tgmm_server_open_lineage")
        self._n_gauss[lid.value] = g.shape[0]
        return lid.value

    def close_lineage(self, lineage: int):
        L.check(L.gmem().tgmm_server_close_lineage(self.h, lineage), "tgmm_server_close_lineage")
        self._n_gauss.pop(lineage, None)

    def read_lineage(self, lineage: int) -> np.ndarray:
        g = np.zeros(self._n_gauss[lineage], L.GAUSS_DTYPE)
        L.check(L.gmem().tgmm_server_read_lineage(self.h, lineage, g.ctypes.data), "tgmm_server_read_lineage")
        return g

    def submit(self, lineage: int, frame, tag: int, want_rnk: bool = True, want_gauss: bool = True,
               compact: bool = False, out=None, runs: bool = False) -> None:
        """frame: an object with query, img, centroids, label_ptr (host arrays of the
        reference layout), e.g. synth.Frame.  With compact=True the voxels go as
        (lin, raw, dims, raw_offset, raw_denom): taken from the frame's attributes of those
        names when present, else from frame.compact().  With runs=True they go as runs
        (run_ptr, run_start, run_len, raw, dims, raw_offset, raw_denom): from the frame's
        attributes of those names when present, else from frame.runs().  The arrays are used
        in place.
        out: optional (rnk, ind, gauss) arrays to receive the outputs (page-locked ones are
        written by the device directly)."""
        if tag in self._pending:
            raise ValueError(f"tag {tag} is already pending")
        ce = np.ascontiguousarray(frame.centroids, np.float32)
        lp = np.ascontiguousarray(frame.label_ptr, np.int64)
        S = lp.shape[0] - 1
        r = L.TgmmServeRequest()
        r.lineage, r.tag = lineage, tag
        r.centroids, r.label_ptr = ce.ctypes.data, lp.ctypes.data
        if runs:
            if hasattr(frame, "run_start"):
                rp, rs, rl, raw, dims, off, den = (frame.run_ptr, frame.run_start, frame.run_len, frame.raw,
                                                   frame.dims, frame.raw_offset, frame.raw_denom)
            else:
                rp, rs, rl, raw, dims, off, den = frame.runs()
            rp = np.ascontiguousarray(rp, np.int32)
            rs = np.ascontiguousarray(rs, np.uint32)
            rl = np.ascontiguousarray(rl, np.uint16)
            raw = np.ascontiguousarray(raw, np.uint16)
            arrs = [rp, rs, rl, raw, ce, lp]
            r.run_ptr, r.run_start, r.run_len, r.raw = rp.ctypes.data, rs.ctypes.data, rl.ctypes.data, raw.ctypes.data
            r.n_runs = rs.shape[0]
            r.dims[:] = list(dims)
            r.raw_offset, r.raw_denom = off, den
            r.n_vox = raw.shape[0]
        elif compact:
            if hasattr(frame, "lin"):
                lin, raw, dims, off, den = frame.lin, frame.raw, frame.dims, frame.raw_offset, frame.raw_denom
            else:
                lin, raw, dims, off, den = frame.compact()
            lin = np.ascontiguousarray(lin, np.uint32)
            raw = np.ascontiguousarray(raw, np.uint16)
            arrs = [lin, raw, ce, lp]
            r.lin, r.raw = lin.ctypes.data, raw.ctypes.data
            r.dims[:] = list(dims)
            r.raw_offset, r.raw_denom = off, den
            r.n_vox = lin.shape[0]
        else:
            q = np.ascontiguousarray(frame.query, np.float32)
            im = np.ascontiguousarray(frame.img, np.float32)
            arrs = [q, im, ce, lp]
            r.query, r.img = q.ctypes.data, im.ctypes.data
            r.n_vox = im.shape[0]
        r.n_sv = S
        pend = _Pending(keep=arrs)
        if want_rnk:
            pend.rnk = out[0][:5 * S] if out is not None else np.zeros(5 * S, np.float32)
            pend.ind = out[1][:5 * S] if out is not None else np.zeros(5 * S, np.int32)
            r.rnk_out, r.ind_out = pend.rnk.ctypes.data, pend.ind.ctypes.data
        if want_gauss and lineage in self._n_gauss:  # (an unknown lineage is answered with an error)
            K = self._n_gauss[lineage]
            pend.gauss = out[2][:K] if out is not None else np.zeros(K, L.GAUSS_DTYPE)
            r.gm_out = pend.gauss.ctypes.data
        self._pending[tag] = pend
        rc = L.gmem().tgmm_server_submit(self.h, C.byref(r))
        if rc:
            del self._pending[tag]
            L.check(rc, "tgmm_server_submit")

    def poll(self, wait_ms: int = 0, max_results: int = 256) -> list[ServeResult]:
        buf = (L.TgmmServeResult * max_results)()
        n = C.c_int32()
        L.check(L.gmem().tgmm_server_poll(self.h, buf, max_results, wait_ms, C.byref(n)), "tgmm_server_poll")
        out = []
        for i in range(n.value):
            b = buf[i]
            pend = self._pending.pop(b.tag, _Pending())
            out.append(ServeResult(tag=b.tag, lineage=b.lineage, status=b.status, stats=_stats(b.stats),
                                   submit_ms=b.submit_ms, start_ms=b.start_ms, done_ms=b.done_ms,
                                   batch_id=b.batch_id, batch_frames=b.batch_frames, rnk=pend.rnk, ind=pend.ind,
                                   gauss=pend.gauss))
        return out

    def drain(self) -> list[ServeResult]:
        """Every outstanding result (blocks until the server has nothing pending)."""
        out = []
        while self._pending:
            got = self.poll(wait_ms=-1)
            if not got:
                break
            out.extend(got)
        return out

    def stats(self) -> dict:
        st = L.TgmmServerStats()
        L.check(L.gmem().tgmm_server_stats(self.h, C.byref(st)), "tgmm_server_stats")
        return {k: getattr(st, k) for k, _ in L.TgmmServerStats._fields_}
