"""The split round on the GPU (tgmm_split_round; mainTrackingGaussianMixtureModel.cpp:1233-1507
with the candidates given): after a first 20-iteration EM, the five Gaussians with the most
supervoxels are split; the local log-likelihoods before and after and the EM on the split
mixture are held to the oracle's restatement of the round run from the same first-EM output
(before: 1e-10 relative, the same inputs; the second EM with test_gpu_em's tolerances; after:
1e-7 relative, since it follows that EM)."""
import ctypes as C

import numpy as np
import pytest

import _fixtures as F
from _parity import compare
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1", "hard"])
def test_split_round_matches_the_oracle(cuda_ok, name):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame(name)
    df = E.to_device(f)
    prm = F.params(20)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss + 5)
    first = plan.run_host(df, f.gauss, prm)
    g = first["gauss"]
    live = np.flatnonzero((g["m_o"][:, 0] > -1e31) & (g["fixed"] == 0))
    cand = [int(k) for k in live[np.argsort(-g["supervoxelNum"][live], kind="stable")[:5]]]
    assert all(g["supervoxelNum"][k] > 0 for k in cand)
    K, n = f.n_gauss, len(cand)
    gh = np.zeros(K + n, L.GAUSS_DTYPE)
    gh[:K] = g
    ind0 = torch.from_numpy(first["ind"]).cuda()
    rnk = torch.empty(5 * f.n_sv, device="cuda")
    ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
    before, after = np.zeros(n), np.zeros(n)
    st = L.TgmmEmStats()
    cf = df.cframe()
    ca = np.asarray(cand, np.int32)
    rc = L.gmem().tgmm_split_round(plan.h, C.byref(cf), gh.ctypes.data, K, ind0.data_ptr(), ca.ctypes.data, n,
                                   rnk.data_ptr(), ind.data_ptr(), C.byref(prm), before.ctypes.data,
                                   after.ctypes.data, C.byref(st), torch.cuda.current_stream().cuda_stream)
    assert rc == L.TGMM_OK, L.gmem().tgmm_last_error()
    plan.close()
    o = O.split_round(f.query, f.img, f.centroids, f.label_ptr, g, first["ind"], cand,
                      O.params(max_iter=20, tol=-1.0))
    np.testing.assert_allclose(before, o["before"], rtol=1e-10)
    got = dict(gauss=gh, rnk=rnk.cpu().numpy(), ind=ind.cpu().numpy(), **E.stats_dict(st))
    compare(got, o)
    np.testing.assert_allclose(after, o["after"], rtol=1e-7)
    assert gh["fixed"][[k for k in range(K) if k not in cand]].all()
    assert not gh["fixed"][cand].any() and not gh["fixed"][K:].any()
