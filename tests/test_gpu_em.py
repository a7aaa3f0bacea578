"""GPU parity: the sm_100a EM against the FP64 oracle on seeded workloads.

Tolerances: kNN candidate lists and supervoxel assignments exact; responsibilities
1e-5 absolute; means 1e-3 voxel; precision matrices 1e-4 relative (to the largest entry
of each matrix); log-likelihood 1e-6 relative with the mixed-precision voxel terms and
1e-9 with FP64 voxel terms.
"""
import numpy as np
import pytest

import _fixtures as F
from _parity import compare
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = ["tiny", "small", "c1", "hard", "big", "moved", "split", "crowded"]


def gpu_run(name, iters=20, tol=-1.0, **kw):
    import torch
    from tgmm_b200 import engine as E
    f = F.frame(name)
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    out = plan.run_host(df, f.gauss, F.params(iters, tol, **kw))
    plan.close()
    torch.cuda.synchronize()
    return out


def oracle_run(name, iters=20, tol=-1.0, ll_mode=O.LL_AS_REFERENCE, mode=O.MODE_FP64):
    f = F.frame(name)
    return O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss,
                    O.params(max_iter=iters, tol=tol, ll_mode=ll_mode, mode=mode))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("iters", [1, 2, 20])
def test_em_matches_fp64_oracle(cuda_ok, name, iters):
    compare(gpu_run(name, iters), oracle_run(name, iters))


def test_knn_lists_and_searches(cuda_ok):
    """After the first iteration a supervoxel's five candidates come from its list of the
    eight nearest Gaussians unless they moved too far, when it searches the grid again;
    the candidates match the oracle's either way (test_em_matches_fp64_oracle), and both
    ways run on these frames."""
    c1 = gpu_run("c1", 20)
    assert 0 <= c1["knn_searches"] < F.frame("c1").n_sv  # most supervoxels never search again
    moved = gpu_run("moved", 20)
    assert moved["knn_searches"] > 0


@pytest.mark.parametrize("name", ["tiny", "hard", "big"])
def test_em_fp64_likelihood(cuda_ok, name):
    from tgmm_b200 import _lib as L
    g = gpu_run(name, 20, ll_precision=L.TGMM_LLPREC_FP64)
    compare(g, oracle_run(name, 20), ll_rtol=1e-9)


@pytest.mark.parametrize("name", ["tiny", "hard", "big"])
@pytest.mark.parametrize("tol", [0.0, 1e-6])
def test_convergence_rule(cuda_ok, name, tol):
    g = gpu_run(name, 50, tol)
    o = oracle_run(name, 50, tol)
    assert g["converged"] == o["converged"] == 1
    compare(g, o)


@pytest.mark.parametrize("name", ["hard", "big"])
def test_true_likelihood_mode(cuda_ok, name):
    from tgmm_b200 import _lib as L
    g = gpu_run(name, 50, 1e-6, ll_mode=L.TGMM_LL_TRUE)
    o = oracle_run(name, 50, 1e-6, ll_mode=O.LL_TRUE)
    compare(g, o)
    assert g["ll"] == g["ll_true"]


def test_knn_standalone_bitexact(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    rng = np.random.default_rng(0)
    for nq, nref in [(1, 5), (37, 5), (1000, 300), (5000, 4000), (20000, 20000)]:
        q = rng.uniform(0, 200, size=(3, nq)).astype(np.float32)
        r = rng.uniform(0, 200, size=(nref, 3)).astype(np.float32)
        # exact duplicates and integer lattice points make distance ties
        if nref > 10:
            r[5:10] = r[0]
            r[10:20] = np.round(r[10:20])
            q[:, :10] = np.round(q[:, :10])
        qf, rf = q.reshape(-1), r.reshape(-1)
        got = E.knn(torch.from_numpy(qf).cuda(), torch.from_numpy(rf).cuda()).cpu().numpy()
        np.testing.assert_array_equal(got, O.knn(qf, rf))


def test_knn_far_and_dead_refs(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    rng = np.random.default_rng(1)
    q = rng.uniform(0, 50, size=(3, 200)).astype(np.float32).reshape(-1)
    r = rng.uniform(0, 50, size=(40, 3)).astype(np.float32)
    r[:36] = -1e32          # dead Gaussians: infinite distance, lowest indices first
    r[36] = [1e6, 1e6, 1e6]  # far but finite
    rf = r.reshape(-1)
    got = E.knn(torch.from_numpy(q).cuda(), torch.from_numpy(rf).cuda()).cpu().numpy()
    np.testing.assert_array_equal(got, O.knn(q, rf))


def test_batch_bitidentical_to_alone(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    names = ["tiny", "small", "hard", "big", "c1"]
    frames = [F.frame(n) for n in names]
    p = F.params(20, -1.0)
    dfs = [E.to_device(f) for f in frames]
    alone = []
    for f, df in zip(frames, dfs):
        plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
        gm = E.gauss_to_device(f.gauss)
        rnk = torch.empty(5 * f.n_sv, device="cuda")
        ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
        plan.run_device(df, gm, rnk, ind, p)
        alone.append((gm.cpu().numpy().copy(), rnk.cpu().numpy(), ind.cpu().numpy()))
        plan.close()
    plan = E.Plan(sum(f.n_vox for f in frames), sum(f.n_sv for f in frames), sum(f.n_gauss for f in frames),
                  max_frames=len(frames))
    gms = [E.gauss_to_device(f.gauss) for f in frames]
    rnks = [torch.empty(5 * f.n_sv, device="cuda") for f in frames]
    inds = [torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda") for f in frames]
    stats = plan.run_batch(dfs, gms, rnks, inds, p)
    from tgmm_b200 import _lib as L
    for i in range(len(frames)):
        got = gms[i].cpu().numpy().view(L.GAUSS_DTYPE)
        want = alone[i][0].view(L.GAUSS_DTYPE)
        diff = [k for k in L.GAUSS_DTYPE.names if not np.array_equal(got[k], want[k])]
        assert not diff, (names[i], diff, [(k, np.argwhere(got[k] != want[k])[:5].tolist()) for k in diff])
        np.testing.assert_array_equal(rnks[i].cpu().numpy(), alone[i][1])
        np.testing.assert_array_equal(inds[i].cpu().numpy(), alone[i][2])
        assert stats[i]["iterations"] == 20
    plan.close()


def test_update_priors_device(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    o = oracle_run("hard", 20)
    g = o["gauss"].copy()
    gm = E.gauss_to_device(g)
    E.update_priors(gm, g.shape[0], 0.01, 1.0, 0.8, -1.0, True)
    got = E.gauss_from_device(gm)
    ref = g.copy()
    lib = O.lib()
    lib.or_update_priors(ref.ctypes.data, ref.shape[0], 0.01, 1.0, 0.8, float(np.sum(g["alpha_k"])))
    for key in ("m_o", "beta_o", "nu_o", "W_o", "alpha_o", "nu_k", "W_k"):
        np.testing.assert_allclose(got[key], ref[key], rtol=1e-12, atol=0)


def test_bad_csr_is_rejected(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame("tiny")
    df = E.to_device(f)
    bad = df.label_ptr.clone()
    bad[3] = bad[4] + 5  # not monotone
    df.label_ptr = bad
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    with pytest.raises(L.TgmmError) as ei:
        plan.run_host(df, f.gauss, F.params(5))
    assert ei.value.code == L.TGMM_ERR_BAD_CSR
    # the plan stays usable
    out = plan.run_host(E.to_device(f), f.gauss, F.params(5))
    assert out["iterations"] == 5
    plan.close()


def test_capacity_and_params_rejected(cuda_ok):
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame("tiny")
    plan = E.Plan(f.n_vox - 1, f.n_sv, f.n_gauss)
    with pytest.raises(L.TgmmError) as ei:
        plan.run_host(E.to_device(f), f.gauss, F.params(5))
    assert ei.value.code == L.TGMM_ERR_BAD_SIZE
    plan.close()
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    p = F.params(5)
    p.lambda_min = -1.0
    with pytest.raises(L.TgmmError) as ei:
        plan.run_host(E.to_device(f), f.gauss, p)
    assert ei.value.code == L.TGMM_ERR_NOT_SET
    plan.close()


def test_page_locked_gaussians_give_the_same_result(cuda_ok):
    """tgmm_em_run reads page-locked Gaussian records with a kernel (so that they do not queue
    behind the caller's uploads on the copy engines) and copies pageable ones: both give the
    same bytes."""
    import ctypes as C
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame("hard")
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    want = plan.run_host(df, f.gauss, F.params(20))
    pinned = torch.from_numpy(L.records(f.gauss).view(np.uint8)).pin_memory()
    rnk = torch.empty(5 * f.n_sv, device="cuda")
    ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
    st = L.TgmmEmStats()
    cf = df.cframe()
    prm = F.params(20)
    rc = L.gmem().tgmm_em_run(plan.h, C.byref(cf), pinned.data_ptr(), rnk.data_ptr(), ind.data_ptr(), None,
                              C.byref(prm), C.byref(st), torch.cuda.current_stream().cuda_stream)
    assert rc == L.TGMM_OK
    plan.close()
    assert L.records_equal(pinned.numpy().view(L.GAUSS_DTYPE), want["gauss"])
    np.testing.assert_array_equal(rnk.cpu().numpy(), want["rnk"])
    np.testing.assert_array_equal(ind.cpu().numpy(), want["ind"])
