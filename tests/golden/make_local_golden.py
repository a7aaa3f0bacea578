"""Generates tests/golden/local_ll.npz by running the REFERENCE's own calculateLocalLikelihood
(UtilsCUDA/GMEMupdateCUDA.cu compiled from its sources by oracle/build_ref.sh) after the
reference's own 20-iteration EM, on seeded test workloads.  Needs a GPU and
oracle/_ref/libtgmm_ref.so.

    python tests/golden/make_local_golden.py [--out DIR]

For each case (c1, hard, big -- big has supervoxels above 1024 voxels) the file holds
  {case}_input_sha256    digest of the frame's inputs (tests/_golden.input_digest)
  {case}_gauss, _ind     the reference EM's records and candidates after 20 iterations
  {case}_list_ptr/_idx   the supervoxel lists: every Gaussian's assigned supervoxels (as the
                         split round forms them, main:1303-1331), the largest supervoxels, a
                         seeded random list with repeats
  {case}_ll              the reference's local log-likelihood of each list"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _fixtures as F  # noqa: E402
from _golden import input_digest  # noqa: E402

CASES = ["c1", "hard", "big"]


def lists_for(f, g, seed):
    rng = np.random.default_rng(seed)
    lists = [[int(s) for s in x["supervoxelIdx"][:x["supervoxelNum"]]] for x in g if x["supervoxelNum"] > 0]
    sizes = np.diff(f.label_ptr)
    lists.append([int(s) for s in np.argsort(-sizes, kind="stable")[:8]])
    lists.append([int(s) for s in rng.integers(0, f.n_sv, size=12)])
    return lists


def main():
    from oracle import oracle as O
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libtgmm_ref.so is missing: run oracle/build_ref.sh where the reference sources are")
    os.makedirs(a.out, exist_ok=True)
    out = {}
    for name in CASES:
        f = F.frame(name)
        assert f.n_sv <= 1024
        r = O.ref_em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, max_iter=20, tol=-1.0)
        lists = lists_for(f, r["gauss"], 17)
        ptr, idx = O.lists_csr(lists)
        out[f"{name}_input_sha256"] = np.array(input_digest(f))
        out[f"{name}_gauss"] = r["gauss"]
        out[f"{name}_ind"] = r["ind"]
        out[f"{name}_list_ptr"] = ptr
        out[f"{name}_list_idx"] = idx
        out[f"{name}_ll"] = O.ref_local_likelihood(f.query, f.img, f.label_ptr, r["ind"], r["gauss"], lists)
        print(f"{name}: S={f.n_sv} K={f.n_gauss} lists={len(lists)}")
    path = os.path.join(a.out, "local_ll.npz")
    np.savez_compressed(path, **out)
    print(f"-> {path} ({os.path.getsize(path)} B)")


if __name__ == "__main__":
    main()
