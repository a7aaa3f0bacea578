"""Generates the frame-preparation golden fixtures in this folder by running the REFERENCE's
own supervoxel trimming and statistics (temporalLogicalRules/supervoxel.cpp) and its erase of
small supervoxels (nucleiChSvWshedPBC/hierarchicalSegmentation.cpp), compiled from their
sources by oracle/build_ref.sh into oracle/_ref/libtgmm_ref_f1.so (host code; no GPU needed),
on the seeded volumes of tests/_volumes.py.

    python tests/golden/make_frame_golden.py [--out DIR]

Each frame_<case>.npz holds:
  input_sha256   digest of the raw and label volumes (pins the generator)
  params         max_size, max_pct, conn, min_size
  thr, cnt       per supervoxel: trimSupervoxel<uint16>()'s threshold and the voxels it keeps
  kept_ptr, kept_lin   the kept voxels' linear indices, CSR over the supervoxels
  cent           per supervoxel: weightedGaussianStatistics<uint16>(true)'s centroid (x, y, z)
  order          the survivors of the size filter in eraseSupervoxelFromCurrentSegmentation's order"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _volumes as V  # noqa: E402

FRAME_CASES = {
    "frame_default": dict(seed=1, max_size=3000, max_pct=0.4, conn=6, min_size=50),
    "frame_conn26": dict(seed=2, max_size=3000, max_pct=0.4, conn=26, min_size=50),
    "frame_big": dict(seed=15, big=True, dims=(160, 144, 40), n_nuclei=80, max_size=3000, max_pct=0.4, conn=6,
                      min_size=50),
}


def volume(case):
    return V.make(seed=case["seed"], **{k: case[k] for k in ("dims", "n_nuclei", "big") if k in case})


def digest(raw, lab) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(raw).tobytes())
    h.update(np.ascontiguousarray(lab).tobytes())
    return h.hexdigest()


def main():
    from oracle import oracle as O
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not O.ref_f1_available():
        raise SystemExit("oracle/_ref/libtgmm_ref_f1.so is missing: run oracle/build_ref.sh where the reference "
                         "sources are")
    for name, c in FRAME_CASES.items():
        raw, lab, n = volume(c)
        ptr, lin = O.supervoxel_lists(lab, n)
        r = O.ref_trim_stats(raw, ptr, lin, c["max_size"], c["max_pct"], c["conn"])
        order = O.ref_erase_order((r["cnt"] < c["min_size"]).astype(np.uint8))
        kept_ptr = np.concatenate([[0], np.cumsum(r["cnt"])]).astype(np.int64)
        kept_lin = np.concatenate(r["lists"]).astype(np.uint32) if n else np.zeros(0, np.uint32)
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), input_sha256=np.array(digest(raw, lab)),
                            params=np.array([c["max_size"], c["max_pct"], c["conn"], c["min_size"]], np.float64),
                            thr=r["thr"], cnt=r["cnt"], kept_ptr=kept_ptr, kept_lin=kept_lin, cent=r["cent"],
                            order=order)
        print(name, n, "supervoxels,", len(order), "kept")


if __name__ == "__main__":
    main()
