"""The local log-likelihood of supervoxel lists (tgmm_local_likelihood; the reference's
calculateLocalLikelihood, GMEMupdateCUDA.cu:2952-3055 with its kernel :1989-2103), the
quantity the split round compares before and after a proposed division.

After a 20-iteration EM on the GPU, the lists are the ones the reference's split round
forms (each Gaussian's assigned supervoxels, main:1303-1331) plus lists with repeated
supervoxels, the frame's largest supervoxels (above 1024 voxels: the reference's per-thread
overwrite) and an empty list.  Held to the FP64 oracle at 1e-10 relative, and to the
reference's own kernels (compiled from its sources, float sums) at 2e-5 relative.
"""
import numpy as np
import pytest

import _fixtures as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _after_em(name):
    import torch
    from tgmm_b200 import engine as E
    f = F.frame(name)
    df = E.to_device(f)
    gm = E.gauss_to_device(f.gauss)
    rnk = torch.empty(5 * f.n_sv, device="cuda")
    ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    plan.run_device(df, gm, rnk, ind, F.params(20))
    plan.close()
    return f, df, gm, ind


def _lists(f, g, seed):
    rng = np.random.default_rng(seed)
    lists = [list(x["supervoxelIdx"][:x["supervoxelNum"]]) for x in g if x["supervoxelNum"] > 0]
    sizes = np.diff(f.label_ptr)
    lists.append(list(np.argsort(-sizes, kind="stable")[:8]))        # the largest supervoxels
    lists.append(list(rng.integers(0, f.n_sv, size=12)))             # random, repeats allowed
    lists.append([int(rng.integers(0, f.n_sv))] * 3)                 # one supervoxel three times
    lists.append([])
    return [[int(s) for s in x] for x in lists]


@pytest.mark.parametrize("name", ["c1", "hard", "big"])
def test_local_likelihood_matches_fp64_oracle(cuda_ok, name):
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f, df, gm, ind = _after_em(name)
    g = gm.cpu().numpy().view(L.GAUSS_DTYPE)
    lists = _lists(f, g, 5)
    if name == "big":
        assert np.diff(f.label_ptr).max() > 1024
    got = E.local_likelihood(df, ind, gm, lists)
    want = O.local_likelihood(f.query, f.img, f.label_ptr, ind.cpu().numpy(), g, lists)
    assert got[-1] == 0.0 and want[-1] == 0.0
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-9)


@pytest.mark.skipif(not O.ref_available(), reason="the reference's GPU path is not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("name", ["c1", "hard", "big"])
def test_local_likelihood_matches_the_reference_kernels(cuda_ok, name):
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f, df, gm, ind = _after_em(name)
    g = gm.cpu().numpy().view(L.GAUSS_DTYPE)
    lists = [x for x in _lists(f, g, 9) if x]
    got = E.local_likelihood(df, ind, gm, lists)
    ref = O.ref_local_likelihood(f.query, f.img, f.label_ptr, ind.cpu().numpy(), g, lists)
    np.testing.assert_allclose(got, ref, rtol=2e-5)
    # the oracle's float-sum mode restates the reference's reductions
    r32 = O.local_likelihood(f.query, f.img, f.label_ptr, ind.cpu().numpy(), g, lists, mode=O.MODE_REF32)
    np.testing.assert_allclose(r32, ref, rtol=1e-6)


def test_local_likelihood_rejects_bad_indices(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f, df, gm, ind = _after_em("tiny")
    with pytest.raises(L.TgmmError) as ei:
        E.local_likelihood(df, ind, gm, [[0, f.n_sv]])
    assert ei.value.code == L.TGMM_ERR_INVALID_ARG
    bad = ind.clone()
    bad[0] = f.n_gauss + 3  # a candidate beyond the Gaussians
    with pytest.raises(L.TgmmError) as ei:
        E.local_likelihood(df, bad, gm, [[0]])
    assert ei.value.code == L.TGMM_ERR_INVALID_ARG
    assert E.local_likelihood(df, ind, gm, [[0]])[0] != 0.0  # usable afterwards
    torch.cuda.synchronize()
