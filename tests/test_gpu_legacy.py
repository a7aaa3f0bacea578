"""A C++ program written against the reference's own interface (tests/legacy_harness.cpp:
GMEMinitializeMemoryWithSupervoxels -> GMEMvariationalInferenceCUDAWithSupervoxels ->
GMEMreleaseMemoryWithSupervoxels, as mainTrackingGaussianMixtureModel.cpp:1065-1107 calls
them), linked against the library, gives the results of the C ABI on the same frame."""
import os
import subprocess

import numpy as np
import pytest

import _fixtures as F
from tgmm_b200 import _lib as L

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


@pytest.mark.parametrize("name", ["small", "hard"])
def test_legacy_entry_points_match_the_c_abi(cuda_ok, tmp_path, name):
    from tgmm_b200 import engine as E
    exe = tmp_path / "legacy"
    r = subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(ROOT, "tests", "legacy_harness.cpp"), "-I" + INC,
                        "-I/usr/local/cuda/include", L.GMEM_SO, "-L/usr/local/cuda/lib64", "-lcudart",
                        "-Wl,-rpath," + os.path.dirname(L.GMEM_SO), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    f = F.frame(name)
    d = tmp_path
    f.query.tofile(d / "query.bin")
    f.img.tofile(d / "img.bin")
    f.centroids.tofile(d / "cent.bin")
    f.label_ptr.tofile(d / "lptr.bin")
    np.ascontiguousarray(f.gauss).tofile(d / "gauss.bin")
    iters, tol = 20, 0.0
    r = subprocess.run([str(exe), str(d), str(iters), str(tol)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Log-likelihood" in r.stdout
    g = np.fromfile(d / "gauss_out.bin", dtype=L.GAUSS_DTYPE)
    rnk = np.fromfile(d / "rnk.bin", dtype=np.float32)
    ind = np.fromfile(d / "ind.bin", dtype=np.int32)
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    want = plan.run_host(df, f.gauss, F.params(iters, tol))
    plan.close()
    np.testing.assert_array_equal(ind, want["ind"])
    np.testing.assert_array_equal(rnk, want["rnk"])
    for k in L.GAUSS_DTYPE.names:
        np.testing.assert_array_equal(g[k], want["gauss"][k], err_msg=k)
    # calculateLocalLikelihood around every Gaussian equals tgmm_local_likelihood bit for bit
    local = np.fromfile(d / "local.bin", dtype=np.float64)
    lists = [list(x["supervoxelIdx"][:x["supervoxelNum"]]) for x in g]
    import torch
    got = E.local_likelihood(df, torch.from_numpy(ind).cuda(), E.gauss_to_device(g), lists)
    empty = np.array([len(x) == 0 for x in lists])
    np.testing.assert_array_equal(local[~empty], got[~empty])
    assert np.all(local[empty] == 0.0)
