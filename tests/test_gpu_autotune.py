"""The kNN/E-step width (lanes per supervoxel) only changes speed: every width gives the
same bits, and the autotuner's choice leaves the results as they are."""
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
        for lanes in (8, 16, 32, 8):
            plan.set_knn_group(lanes)
            runs.setdefault(lanes, []).append(plan.run_host(df, f.gauss, F.params(20, -1.0)))
    finally:
        plan.close()
    same(runs[8][0], runs[8][1])
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
        assert lanes in (8, 16, 32)
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
        with pytest.raises(L.TgmmError):
            plan.set_knn_group(4)
    finally:
        plan.close()
