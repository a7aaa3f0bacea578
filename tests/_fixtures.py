"""Seeded workloads shared by the tests (inputs are generated, never read from outside)."""
from __future__ import annotations

import functools

import numpy as np

from tgmm_b200 import _lib as L
from tgmm_b200 import synth

SPEC_HARD = synth.VolumeSpec(dims=(96, 96, 48), n_nuclei=40, axis_min=3.0, axis_max=7.0, jitter=3.0)
SPEC_BIG = synth.VolumeSpec(dims=(96, 96, 48), n_nuclei=6, axis_min=11.0, axis_max=14.0)
SPEC_SMALL = synth.VolumeSpec(dims=(128, 128, 48), n_nuclei=60, axis_min=3.0, axis_max=6.0)


def _perturb(frame, seed):
    """Harder Gaussian sets: duplicated Gaussians (soft responsibilities, Gaussians that
    die), a fixed Gaussian, one dead from the start, anisotropic precisions."""
    rng = np.random.default_rng(seed)
    g = frame.gauss.copy()
    K = g.shape[0]
    g["W_k"][:, 0] *= rng.uniform(0.6, 1.6, K)
    g["W_k"][:, 3] *= rng.uniform(0.6, 1.6, K)
    g["W_k"][:, 1] = 0.2 * np.sqrt(g["W_k"][:, 0] * g["W_k"][:, 3]) * rng.uniform(-1, 1, K)
    dup = rng.choice(K, size=max(1, K // 4), replace=False)
    extra = g[dup].copy()
    extra["m_k"] += rng.normal(0, 2.5, size=(dup.size, 3))
    extra["m_o"] = extra["m_k"]
    extra["alpha_k"] *= 0.5
    extra["alpha_o"] = 1e-3  # these lose their supervoxels and die through alpha/sum(alpha) < 1e-5
    twins = g[rng.choice(K, size=3, replace=False)].copy()  # near-copies: split responsibilities
    twins["m_k"] += rng.normal(0, 0.004, size=(3, 3))
    g = np.concatenate([g, extra, twins]).astype(L.GAUSS_DTYPE)
    g["fixed"][1] = 1
    dead = 2
    g["m_o"][dead] = -1e32
    g["m_k"][dead] = -1e32
    g["alpha_k"][dead] = 0.0
    g["W_k"][dead] = [1, 0, 0, 1, 0, 1]
    frame.gauss = g
    return frame


def _displace(frame, seed, sigma=3.0):
    """Every Gaussian (mean and prior mean) starts sigma voxels off its nucleus: the first
    iterations move them by voxels, so the supervoxels' kNN neighbour lists go stale and
    are searched again."""
    rng = np.random.default_rng(seed)
    g = frame.gauss.copy()
    shift = rng.normal(0, sigma, size=(g.shape[0], 3))
    g["m_k"] += shift
    g["m_o"] += shift
    frame.gauss = g
    return frame


def _split(frame, piece=12):
    """Every supervoxel cut into consecutive pieces of `piece` voxels (the last piece takes
    the rest), each piece a supervoxel with its FP32 intensity-weighted centroid: each
    Gaussian becomes a candidate of many small supervoxels (more than the 32 pairs of its
    M-step bucket) and takes more than 32 of them (rnk > 0.5), so both ordered-scan
    branches run."""
    lp = frame.label_ptr
    cuts = [0]
    for s in range(frame.n_sv):
        a, b = int(lp[s]), int(lp[s + 1])
        p = a + piece
        while p < b:
            if b - p < piece // 2:
                break
            cuts.append(p)
            p += piece
        cuts.append(b)
    cuts = np.array(sorted(set(cuts)), np.int64)
    N = frame.n_vox
    q = frame.query.reshape(3, N).astype(np.float64)
    w = frame.img.astype(np.float64)
    sw = np.add.reduceat(w, cuts[:-1])
    cent = np.stack([np.add.reduceat(q[d] * w, cuts[:-1]) / sw for d in range(3)]).astype(np.float32)
    frame.label_ptr = cuts
    frame.centroids = np.ascontiguousarray(cent.reshape(-1))
    frame.sv_nucleus = np.zeros(cuts.size - 1, np.int32)
    return frame


def _crowd(frame, seed, n_copies=40, sigma=0.05):
    """n_copies near-copies of Gaussian 0 within sigma voxels of it: more centres in one
    kNN grid cell than the cell holds (32), so the frame's kNN scans every Gaussian."""
    rng = np.random.default_rng(seed)
    g = frame.gauss.copy()
    extra = np.repeat(g[:1], n_copies)
    extra["m_k"] += rng.normal(0, sigma, size=(n_copies, 3))
    extra["m_o"] = extra["m_k"]
    frame.gauss = np.concatenate([g, extra]).astype(L.GAUSS_DTYPE)
    return frame


@functools.lru_cache(maxsize=None)
def frame(name: str):
    if name == "tiny":
        return synth.generate(synth.TINY, seed=7)
    if name == "small":
        return synth.generate(SPEC_SMALL, seed=3)
    if name == "c1":
        return synth.generate(synth.C1, seed=1)
    if name == "hard":
        return _perturb(synth.generate(SPEC_HARD, seed=11), 11)
    if name == "big":
        return synth.generate(SPEC_BIG, seed=5)
    if name == "moved":
        return _displace(synth.generate(SPEC_SMALL, seed=21), 21)
    if name == "split":
        return _split(synth.generate(SPEC_SMALL, seed=31))
    if name == "crowded":
        return _crowd(synth.generate(SPEC_SMALL, seed=41), 41)
    raise KeyError(name)


def params(iters=20, tol=-1.0, **kw):
    """EM parameters of the workloads; tol < 0 runs exactly `iters` iterations."""
    return synth.em_params(iters=iters, tol=tol, **kw)
