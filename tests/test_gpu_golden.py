"""The CUDA path against the reference's own outputs (tests/golden): the same kNN sets,
survivors and supervoxel assignments, and values within the reference's FP32 error of
it (responsibilities <= 1e-4, means <= 1e-3 voxel, precision matrices <= 5e-3 relative;
the FP64 oracle sits at the same distance from the reference, and the CUDA path is held
to 1e-5 / 1e-3 / 1e-4 of the FP64 oracle by test_gpu_em.py)."""
import numpy as np
import pytest

import _fixtures as F
import _golden as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("it", G.ITERS)
@pytest.mark.parametrize("name", G.CASES)
def test_cuda_path_matches_reference_outputs(cuda_ok, name, it):
    from tgmm_b200 import engine as E
    z, f = G.load(name), F.frame(name)
    assert str(z["input_sha256"]) == G.input_digest(f)
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        out = plan.run_host(df, f.gauss, F.params(it, -1.0))
    finally:
        plan.close()
    G.compare_with_reference(z, it, out, f.n_sv, rnk_tol=1e-4, m_tol=1e-3, w_rtol=5e-3, same_slot_order=False)


@pytest.mark.parametrize("name", G.CASES)
def test_cuda_knn_sets_match_reference(cuda_ok, name):
    import torch
    from tgmm_b200 import engine as E
    z, f = G.load(name), F.frame(name)
    q = torch.from_numpy(f.centroids).cuda()
    r = torch.from_numpy(np.ascontiguousarray(f.gauss["m_k"].astype(np.float32)).reshape(-1)).cuda()
    got = E.knn(q, r).cpu().numpy()
    S = f.n_sv
    np.testing.assert_array_equal(np.sort(got.reshape(5, S), 0), np.sort(z["knn_ind"].reshape(5, S), 0))
