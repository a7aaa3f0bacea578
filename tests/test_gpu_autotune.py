"""The kNN/E-step width (lanes per supervoxel) and whether the voxel pass runs the next
iteration's kNN/E-step only change speed: every choice gives the same bits, and the
autotuner's choices leave the results as they are."""
import numpy as np
import pytest

import _fixtures as F
from tgmm_b200 import _lib as L

pytestmark = pytest.mark.gpu


def same(a, b):
    np.testing.assert_array_equal(a["ind"], b["ind"])
    np.testing.assert_array_equal(a["rnk"], b["rnk"])
    for k in L.GAUSS_DTYPE.names:
        np.testing.assert_array_equal(a["gauss"][k], b["gauss"][k], err_msg=k)
    assert a["ll"] == b["ll"] and a["iterations"] == b["iterations"]


@pytest.mark.parametrize("name", ["c1", "hard", "big"])
def test_every_width_gives_the_same_bits(cuda_ok, name):
    from tgmm_b200 import engine as E
    f = F.frame(name)
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        runs = {}
        for lanes in (8, 4, 16, 32, 8):
            plan.set_knn_group(lanes)
            runs.setdefault(lanes, []).append(plan.run_host(df, f.gauss, F.params(20, -1.0)))
    finally:
        plan.close()
    same(runs[8][0], runs[8][1])
    same(runs[8][0], runs[4][0])
    same(runs[8][0], runs[16][0])
    same(runs[8][0], runs[32][0])


def test_autotune_keeps_the_results(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    names = ["c1", "small", "hard"]
    fr = [F.frame(n) for n in names]
    dfs = [E.to_device(f) for f in fr]
    gm0 = [E.gauss_to_device(f.gauss) for f in fr]
    prm = F.params(20, -1.0)

    def run(plan):
        gms = [g.clone() for g in gm0]
        rnks = [torch.empty(5 * f.n_sv, device="cuda") for f in fr]
        inds = [torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda") for f in fr]
        st = plan.run_batch(dfs, gms, rnks, inds, prm)
        return [dict(rnk=r.cpu().numpy(), ind=i.cpu().numpy(), gauss=E.gauss_from_device(g), **s)
                for r, i, g, s in zip(rnks, inds, gms, st)], (gms, rnks, inds)

    cap = (sum(f.n_vox for f in fr), sum(f.n_sv for f in fr), sum(f.n_gauss for f in fr))
    plain = E.Plan(*cap, max_frames=len(fr))
    tuned = E.Plan(*cap, max_frames=len(fr))
    try:
        want, _ = run(plain)
        gms = [g.clone() for g in gm0]
        rnks = [torch.empty(5 * f.n_sv, device="cuda") for f in fr]
        inds = [torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda") for f in fr]
        lanes = tuned.autotune(dfs, gms, rnks, inds, prm, reps=2)
        assert lanes in (4, 8, 16, 32)
        for g, g0 in zip(gms, gm0):  # the autotuner only reads the Gaussians
            assert torch.equal(g, g0)
        got, _ = run(tuned)
    finally:
        plain.close()
        tuned.close()
    for a, b in zip(got, want):
        same(a, b)


def test_bad_width_is_refused(cuda_ok):
    from tgmm_b200 import engine as E
    f = F.frame("tiny")
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        for bad in (2, 6, 64):
            with pytest.raises(L.TgmmError):
                plan.set_knn_group(bad)
        # groups of 4 lanes always run the kNN/E-step in its own kernel
        plan.set_knn_group(4)
        plan.set_knn_fusion(True)
        assert plan.tuning() == {"knn_lanes": 4, "knn_fused": False}
    finally:
        plan.close()


@pytest.mark.parametrize("name,tol", [("c1", -1.0), ("hard", -1.0), ("moved", -1.0), ("c1", 1e-6), ("hard", 0.0),
                                      ("moved", 1e-6)])
def test_knn_in_voxel_pass_gives_the_same_bits(cuda_ok, name, tol):
    """The voxel pass running the next iteration's kNN/E-step gives the bits of the two
    kernels one after the other, also when a frame converges and the kNN/E-step it ran
    ahead is dropped (tol >= 0), at every width; groups of 4 lanes keep their own kernel
    whatever the fusion setting."""
    from tgmm_b200 import engine as E
    f = F.frame(name)
    df = E.to_device(f)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        runs = {}
        for lanes in (8, 4, 32):
            plan.set_knn_group(lanes)
            for fused in (False, True, False):
                plan.set_knn_fusion(fused)
                runs.setdefault((lanes, fused), []).append(plan.run_host(df, f.gauss, F.params(30, tol)))
        assert plan.tuning() == {"knn_lanes": 32, "knn_fused": False}
    finally:
        plan.close()
    ref = runs[(8, False)][0]
    if tol >= 0:
        assert ref["converged"] == 1 and ref["iterations"] < 30  # the dropped run-ahead is exercised
    for rs in runs.values():
        for r in rs:
            same(ref, r)


def test_autotune_reads_the_gaussians_only_and_keeps_the_results(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    f = F.frame("c1")
    df = E.to_device(f)
    gm = E.gauss_to_device(f.gauss)
    before = gm.clone()
    rnk = torch.empty(5 * f.n_sv, device="cuda")
    ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        lanes = plan.autotune([df], [gm], [rnk], [ind], F.params(20, -1.0), reps=1)
        torch.cuda.synchronize()
        assert torch.equal(gm, before)
        t = plan.tuning()
        assert t["knn_lanes"] == lanes and isinstance(t["knn_fused"], bool)
        got = plan.run_host(df, f.gauss, F.params(20, -1.0))
        plan.set_knn_group(8)
        plan.set_knn_fusion(False)
        want = plan.run_host(df, f.gauss, F.params(20, -1.0))
    finally:
        plan.close()
    same(got, want)
