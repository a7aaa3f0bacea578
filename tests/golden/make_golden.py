"""Generates the golden fixtures in this folder by running the REFERENCE's own GPU EM
(UtilsCUDA/GMEMupdateCUDA.cu + knnCuda.cu compiled from its sources by oracle/build_ref.sh)
on the seeded test workloads.  Needs a GPU and oracle/_ref/libtgmm_ref.so.

    python tests/golden/make_golden.py [--out DIR]

Each <case>.npz holds, for the inputs that tests/_fixtures.py regenerates from its seed:
  input_sha256   digest of every input array (pins the generator: a changed generator
                 must regenerate the fixtures)
  knn_ind        knnCUDAinPlace on the initial means (reference slot order), J*S int32
  em{I}_gauss    the 288-byte records after GMEMvariationalInferenceCUDAWithSupervoxels
                 with maxIterEM = I and tol < 0 (exactly I iterations), I in ITERS
  em{I}_rnk      rnkCUDA (J*S float32), em{I}_ind  indCUDA (J*S int32)
Only frames with at most 1024 supervoxels are run (the reference's kNN kernel calls
__syncthreads() after an early return of surplus threads)."""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _fixtures as F  # noqa: E402
from _golden import CASES, ITERS, input_digest  # noqa: E402


def main():
    from oracle import oracle as O
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libtgmm_ref.so is missing: run oracle/build_ref.sh where the reference sources are")
    os.makedirs(a.out, exist_ok=True)
    for name in CASES:
        f = F.frame(name)
        assert f.n_sv <= 1024
        out = dict(input_sha256=np.array(input_digest(f)))
        ref_xyz = np.ascontiguousarray(f.gauss["m_k"].astype(np.float32)).reshape(-1)
        out["knn_ind"] = O.ref_knn(f.centroids, ref_xyz)
        for it in ITERS:
            r = O.ref_em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, max_iter=it, tol=-1.0)
            out[f"em{it}_gauss"] = r["gauss"]
            out[f"em{it}_rnk"] = r["rnk"]
            out[f"em{it}_ind"] = r["ind"]
        path = os.path.join(a.out, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: N={f.n_vox} S={f.n_sv} K={f.n_gauss} -> {path} ({os.path.getsize(path)} B)")


if __name__ == "__main__":
    main()
