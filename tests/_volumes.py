"""Seeded synthetic volumes for the frame-preparation tests: a raw 16-bit image of blurred
nuclei over a noisy background and the label volume of an (untrimmed) segmentation, each
supervoxel reaching past its nucleus into the background the way a hierarchical segmentation
at tau does.  Besides ordinary nuclei it plants the cases trimming has to get right:
oversegmented nuclei (two labels), bright islands not connected to a supervoxel's peak,
supervoxels below the minimum size, a flat supervoxel (Otsu degenerate, nothing above its
threshold), a supervoxel joined only across the x border (linear-index neighbours wrap to the
next row) and label numbers with no voxels."""
from __future__ import annotations

import numpy as np


def make(dims=(96, 80, 24), n_nuclei=24, seed=0, background=100.0, specials=True, big=False):
    """Returns (raw (Z, Y, X) uint16, label (Z, Y, X) uint32, n_labels).  big: one more
    supervoxel whose bounding box (70 x 60 x 16 voxels) is larger than a trimming block holds in
    shared memory, around a bright blob (needs dims of at least 72 x 62 x 18)."""
    X, Y, Z = dims
    rng = np.random.default_rng(seed)
    raw = rng.poisson(background, size=(Z, Y, X)).astype(np.float64)
    label = np.zeros((Z, Y, X), np.uint32)
    best = np.full((Z, Y, X), np.inf)
    nxt = 1
    for _ in range(n_nuclei):
        c = np.array([rng.uniform(4, X - 5), rng.uniform(4, Y - 5), rng.uniform(2, Z - 3)])
        ax = np.array([rng.uniform(3.0, 6.5), rng.uniform(3.0, 6.5), rng.uniform(1.5, 3.0)])
        peak = rng.uniform(150.0, 1200.0)
        lo = np.maximum(0, np.floor(c - 1.6 * ax).astype(int))
        hi = np.minimum([X, Y, Z], np.ceil(c + 1.6 * ax).astype(int) + 1)
        zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                                 indexing="ij")
        d = np.sqrt(((xx - c[0]) / ax[0]) ** 2 + ((yy - c[1]) / ax[1]) ** 2 + ((zz - c[2]) / ax[2]) ** 2)
        sl = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
        raw[sl] += peak * np.exp(-0.5 * (1.6 * d) ** 2)
        if specials and rng.random() < 0.3:
            # a bright island in the supervoxel's fringe, apart from its body
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            p = c + 1.3 * ax * u
            di = np.sqrt(((xx - p[0]) / 0.8) ** 2 + ((yy - p[1]) / 0.8) ** 2 + ((zz - p[2]) / 0.6) ** 2)
            raw[sl] += 0.9 * peak * np.exp(-0.5 * di ** 2) * (di < 1.5)
        region = d < 1.5
        closer = region & (d < best[sl])
        labs = np.full(d.shape, nxt, np.uint32)
        if rng.random() < 0.3:  # oversegmented: two supervoxels split by a plane
            labs[(xx - c[0]) * rng.normal() + (yy - c[1]) * rng.normal() > 0] = nxt + 1
            nxt += 2
        else:
            nxt += 1
        label[sl][closer] = labs[closer]
        best[sl][closer] = d[closer]
    if specials:
        # small supervoxels (erased by the size filter)
        for _ in range(3):
            x0, y0, z0 = rng.integers(0, X - 3), rng.integers(0, Y - 3), rng.integers(0, Z - 2)
            free = label[z0:z0 + 2, y0:y0 + 3, x0:x0 + 3] == 0
            raw[z0:z0 + 2, y0:y0 + 3, x0:x0 + 3][free] += 400.0
            label[z0:z0 + 2, y0:y0 + 3, x0:x0 + 3][free] = nxt
            nxt += 1
        # a flat supervoxel: every value equal, nothing strictly above the threshold
        x0, y0, z0 = X // 2, 1, 0
        blk = (slice(z0, z0 + 3), slice(y0, y0 + 5), slice(x0, x0 + 5))
        raw[blk] = 500.0
        label[blk] = nxt
        nxt += 1
        # a supervoxel whose two bright halves meet only across the x border ((X-1, y) + 1 is
        # (0, y+1)), each with a dim fringe so that Otsu's threshold keeps both halves
        z0, y0 = Z // 2, Y // 2
        for z in range(z0, z0 + 5):
            label[z, y0:y0 + 6, X - 3:X] = nxt
            label[z, y0 + 1:y0 + 7, 0:3] = nxt
            raw[z, y0:y0 + 6, X - 3:X - 1] = 300.0
            raw[z, y0 + 1:y0 + 7, 1:3] = 300.0
            raw[z, y0:y0 + 6, X - 1] = 950.0 + rng.integers(0, 40, size=6)
            raw[z, y0 + 1:y0 + 7, 0] = 900.0 + rng.integers(0, 40, size=6)
        nxt += 1
        nxt += 2  # label numbers with no voxels
    if big:
        blk = (slice(1, 17), slice(1, 61), slice(1, 71))
        zz, yy, xx = np.meshgrid(np.arange(1, 17), np.arange(1, 61), np.arange(1, 71), indexing="ij")
        d2 = ((xx - 30.0) / 9.0) ** 2 + ((yy - 25.0) / 8.0) ** 2 + ((zz - 8.0) / 4.0) ** 2
        raw[blk] += 900.0 * np.exp(-0.5 * d2)
        label[blk] = nxt
        nxt += 1
    n_labels = nxt - 1
    # number the supervoxels in an order unrelated to space
    perm = np.concatenate([[0], rng.permutation(n_labels) + 1]).astype(np.uint32)
    label = perm[label]
    raw = np.clip(np.rint(raw), 0, 65535).astype(np.uint16)
    return raw, label, n_labels
