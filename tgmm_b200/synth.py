"""Seeded synthetic nuclei volumes, supervoxels and Gaussian initialisations.

The workloads are the five configurations of the benchmark: a small CPU-runnable frame,
a 1-Gvoxel frame, a batch of 64 uneven volumes, and two served time series.  No public
dataset is involved; every array is generated from a seed by ``libtgmm_synth.so``
(nucleus model, Poisson noise, 26-connected supervoxels inside each nucleus's
anisotropy-scaled Voronoi cell, first-frame Gaussians as TGMM initialises them).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class VolumeSpec:
    dims: tuple            # (X, Y, Z)
    n_nuclei: int
    axis_min: float = 4.0
    axis_max: float = 8.0
    anisotropy: float = 2.0
    peak_min: float = 400.0
    peak_max: float = 1200.0
    background: float = 100.0
    threshold: float = 150.0
    jitter: float = 1.5
    min_size: int = 50

    def cconfig(self) -> L.TgmmSynthConfig:
        c = L.TgmmSynthConfig()
        c.dims[:] = [int(d) for d in self.dims]
        c.axis_min, c.axis_max, c.anisotropy = self.axis_min, self.axis_max, self.anisotropy
        c.peak_min, c.peak_max = self.peak_min, self.peak_max
        c.background, c.threshold, c.jitter, c.min_size = self.background, self.threshold, self.jitter, self.min_size
        return c


# The EM parameters every configuration uses: 20 fixed iterations, W4DOF, scale (1,1,2),
# the reference's regularisation constants.
EM_ITERS = 20


def em_params(iters: int = EM_ITERS, tol: float = 0.0, **kw) -> L.TgmmEmParams:
    p = L.default_params(max_iter_em=iters, tol_likelihood=tol, scale=(1.0, 1.0, 2.0))
    for k, v in kw.items():
        if k in ("scale", "reg_scale"):
            getattr(p, k)[:] = list(v)
        else:
            setattr(p, k, v)
    return p


C1 = VolumeSpec(dims=(256, 256, 64), n_nuclei=300, axis_min=3.0, axis_max=6.0)
C2 = VolumeSpec(dims=(2048, 1024, 512), n_nuclei=20000, axis_min=4.0, axis_max=8.0)
TINY = VolumeSpec(dims=(64, 64, 32), n_nuclei=12, axis_min=3.0, axis_max=5.0)


@dataclass
class Nuclei:
    centre: np.ndarray  # (n,3) float32, voxel coordinates x,y,z
    axes: np.ndarray    # (n,3) semi-axes (z already divided by anisotropy)
    rot: np.ndarray     # (n,9) row-major rotation
    peak: np.ndarray    # (n,)

    @property
    def n(self):
        return self.centre.shape[0]


def random_nuclei(spec: VolumeSpec, seed: int) -> Nuclei:
    n = spec.n_nuclei
    centre = np.zeros((n, 3), np.float32)
    axes = np.zeros((n, 3), np.float32)
    rot = np.zeros((n, 9), np.float32)
    peak = np.zeros((n,), np.float32)
    L.synth().tgmm_synth_nuclei(C.byref(spec.cconfig()), n, seed, L.ptr(centre), L.ptr(axes), L.ptr(rot),
                                L.ptr(peak))
    return Nuclei(centre, axes, rot, peak)


@dataclass
class Frame:
    """One time point in the reference's input layout (host arrays)."""
    query: np.ndarray       # (3*N,) float32, SoA x|y|z
    img: np.ndarray         # (N,) float32 in (0,1]
    centroids: np.ndarray   # (3*S,) float32, SoA
    label_ptr: np.ndarray   # (S+1,) int64
    sv_nucleus: np.ndarray  # (S,) int32
    max_fg: float
    spec: VolumeSpec = None
    nuclei: Nuclei = None
    gauss: np.ndarray = None            # (K,) GAUSS_DTYPE
    gauss_nucleus: np.ndarray = None    # (K,) int32
    meta: dict = field(default_factory=dict)
    raw: np.ndarray = None              # (N,) uint16 foreground values (img = (raw - thr)/(max_fg - thr))

    def compact(self):
        """The frame's voxels as (linear index uint32, raw uint16, dims, offset, denominator):
        6 bytes per voxel that expand exactly into query and img (x = lin % X, y = lin / X
        % Y, z = lin / (X Y); img = float((raw - offset) / denominator) in double)."""
        X, Y, Z = self.spec.dims
        n = self.n_vox
        q = self.query
        lin = (q[:n].astype(np.int64) + X * (q[n:2 * n].astype(np.int64) + Y * q[2 * n:].astype(np.int64)))
        thr = float(np.float32(self.spec.threshold))
        return lin.astype(np.uint32), self.raw, (X, Y, Z), thr, float(self.max_fg) - thr

    def runs(self):
        """The frame's voxels as runs (see runs_of): (run_ptr int32 [S+1], run_start uint32,
        run_len uint16, raw uint16, dims, offset, denominator), about 3 bytes per voxel."""
        lin, raw, dims, off, den = self.compact()
        rp, rs, rl = runs_of(lin, self.label_ptr)
        return rp, rs, rl, raw, dims, off, den

    @property
    def n_vox(self):
        return int(self.img.shape[0])

    @property
    def n_sv(self):
        return int(self.label_ptr.shape[0] - 1)

    @property
    def n_gauss(self):
        return int(self.gauss.shape[0]) if self.gauss is not None else 0


def runs_of(lin: np.ndarray, label_ptr: np.ndarray, max_len: int = 65535):
    """Runs of consecutive linear indices, supervoxel by supervoxel (label_ptr, ascending
    voxels within each): a run starts at a supervoxel's first voxel, after a gap in the
    indices, and every max_len voxels.  Returns run_ptr (int32, S+1: the runs of supervoxel s
    are run_ptr[s] .. run_ptr[s+1]), run_start (uint32) and run_len (uint16)."""
    lin = np.asarray(lin).astype(np.int64)
    lp = np.asarray(label_ptr, np.int64)
    n = lin.shape[0]
    S = lp.shape[0] - 1
    start = np.ones(n, bool)
    start[1:] = lin[1:] != lin[:-1] + 1
    start[lp[:-1][lp[:-1] < n]] = True
    # split runs longer than max_len: the position within its run of every voxel
    idx = np.flatnonzero(start)
    pos = np.arange(n) - np.repeat(idx, np.diff(np.append(idx, n)))
    start |= (pos % max_len == 0)
    idx = np.flatnonzero(start)
    run_len = np.diff(np.append(idx, n))
    run_ptr = np.searchsorted(idx, lp, side="left").astype(np.int32)
    return run_ptr, lin[idx].astype(np.uint32), run_len.astype(np.uint16)


def make_frame(spec: VolumeSpec, nuclei: Nuclei, seed: int) -> Frame:
    lib = L.synth()
    cfg = spec.cconfig()
    h = lib.tgmm_synth_frame(C.byref(cfg), nuclei.n, L.ptr(nuclei.centre), L.ptr(nuclei.axes), L.ptr(nuclei.rot),
                             L.ptr(nuclei.peak), seed)
    try:
        n = lib.tgmm_synth_n_vox(h)
        s = lib.tgmm_synth_n_sv(h)
        q = np.empty(3 * n, np.float32)
        img = np.empty(n, np.float32)
        cent = np.empty(3 * s, np.float32)
        lptr = np.empty(s + 1, np.int64)
        svn = np.empty(s, np.int32)
        lib.tgmm_synth_copy(h, L.ptr(q), L.ptr(img), L.ptr(cent), L.ptr(lptr), L.ptr(svn))
        raw = np.empty(n, np.uint16)
        lib.tgmm_synth_copy_raw(h, L.ptr(raw))
        mx = lib.tgmm_synth_max_fg(h)
    finally:
        pass
    f = Frame(q, img, cent, lptr, svn, float(mx), spec=spec, nuclei=nuclei)
    f.raw = raw
    f.meta["handle"] = h
    return f


def init_gaussians(frame: Frame, seed: int, params: L.TgmmEmParams = None) -> Frame:
    lib = L.synth()
    params = params or em_params()
    h = frame.meta["handle"]
    cfg = frame.spec.cconfig()
    nuc = frame.nuclei
    K = lib.tgmm_synth_init_gaussians(h, C.byref(cfg), nuc.n, L.ptr(nuc.centre), seed, C.byref(params), None, None)
    g = np.zeros(K, L.GAUSS_DTYPE)
    gn = np.zeros(K, np.int32)
    lib.tgmm_synth_init_gaussians(h, C.byref(cfg), nuc.n, L.ptr(nuc.centre), seed, C.byref(params), L.ptr(g),
                                  L.ptr(gn))
    frame.gauss = g
    frame.gauss_nucleus = gn
    return frame


def release(frame: Frame):
    h = frame.meta.pop("handle", None)
    if h:
        L.synth().tgmm_synth_free(h)


def generate(spec: VolumeSpec, seed: int, params: L.TgmmEmParams = None) -> Frame:
    """Nuclei, volume, supervoxels and first-frame Gaussians for one seeded frame."""
    nuclei = random_nuclei(spec, seed)
    f = make_frame(spec, nuclei, seed)
    init_gaussians(f, seed, params)
    release(f)
    return f


def evolve_nuclei(nuc: Nuclei, spec: VolumeSpec, rng: np.random.Generator, sigma: float = 1.5,
                  divide_frac: float = 0.01, offset: float = 3.0) -> Nuclei:
    """One time step: Brownian motion, then a fraction of nuclei divide into two daughters
    placed +/- offset voxels along a random axis (peak, size and orientation kept)."""
    c = nuc.centre + rng.normal(0.0, sigma, nuc.centre.shape).astype(np.float32)
    hi = np.array(spec.dims, np.float32) - 1.0
    c = np.clip(c, 0.0, hi)
    n = c.shape[0]
    div = rng.random(n) < divide_frac
    if not div.any():
        return Nuclei(c, nuc.axes.copy(), nuc.rot.copy(), nuc.peak.copy())
    d = rng.normal(size=(int(div.sum()), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = (d * offset).astype(np.float32)
    c2 = c.copy()
    c2[div] = np.clip(c[div] + d, 0.0, hi)
    extra = np.clip(c[div] - d, 0.0, hi)
    return Nuclei(np.concatenate([c2, extra]), np.concatenate([nuc.axes, nuc.axes[div]]),
                  np.concatenate([nuc.rot, nuc.rot[div]]), np.concatenate([nuc.peak, nuc.peak[div]]))


def batch_specs(n_volumes: int, seed: int):
    """Uneven volumes: dims uniform in [128..512]x[128..512]x[64..128], one nucleus per
    ~3000 voxels clipped to [100, 5000]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_volumes):
        X = int(rng.integers(128, 513))
        Y = int(rng.integers(128, 513))
        Z = int(rng.integers(64, 129))
        n = int(np.clip(round(X * Y * Z / 3000), 100, 5000))
        out.append(VolumeSpec(dims=(X, Y, Z), n_nuclei=n))
    return out


def time_series_iter(spec: VolumeSpec, seed: int, n_frames: int, sigma: float = 1.5, divide_frac: float = 0.01,
                     params: L.TgmmEmParams = None):
    """The frames of time_series one at a time (a consumer can keep a smaller form of each)."""
    rng = np.random.default_rng(seed)
    nuc = random_nuclei(spec, seed)
    f0 = make_frame(spec, nuc, seed * 1000)
    init_gaussians(f0, seed, params)
    release(f0)
    yield f0
    for t in range(1, n_frames):
        nuc = evolve_nuclei(nuc, spec, rng, sigma=sigma, divide_frac=divide_frac)
        f = make_frame(spec, nuc, seed * 1000 + t)
        release(f)
        yield f


def time_series(spec: VolumeSpec, seed: int, n_frames: int, sigma: float = 1.5, divide_frac: float = 0.01,
                params: L.TgmmEmParams = None) -> list:
    """A lineage: frame 0 with first-frame Gaussians, then frames whose nuclei move by
    Brownian steps and divide (evolve_nuclei); later frames carry no Gaussians -- the
    posterior of the previous frame is their prior."""
    return list(time_series_iter(spec, seed, n_frames, sigma=sigma, divide_frac=divide_frac, params=params))
