"""The served form (tgmm_serve.h) on the GPU: every frame's result in the mix of lineages
and batches is bit-identical to the same lineage run alone through tgmm_em_run_device +
tgmm_update_priors; admission against a small HBM budget; answers for frames that can
never run; a two-frame lineage against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

import _fixtures as F
from tgmm_b200 import _lib as L
from tgmm_b200 import synth

pytestmark = pytest.mark.gpu

SPECS = [synth.VolumeSpec(dims=(64, 64, 32), n_nuclei=12, axis_min=3.0, axis_max=5.0),
         synth.VolumeSpec(dims=(96, 96, 48), n_nuclei=30, axis_min=3.0, axis_max=6.0),
         synth.VolumeSpec(dims=(128, 128, 48), n_nuclei=60, axis_min=3.0, axis_max=6.0),
         synth.VolumeSpec(dims=(80, 64, 40), n_nuclei=20, axis_min=3.0, axis_max=5.0)]
N_FRAMES = 4


def lineages():
    return [synth.time_series(spec, seed=100 + i, n_frames=N_FRAMES, divide_frac=0.05) for i, spec in enumerate(SPECS)]


def params(tol=1e-6):
    return F.params(iters=20, tol=tol)


def run_alone(frames, prm):
    """The lineage frame after frame through the plain device API."""
    import torch
    from tgmm_b200 import engine as E
    K = frames[0].n_gauss
    plan = E.Plan(max(f.n_vox for f in frames), max(f.n_sv for f in frames), K)
    gm = E.gauss_to_device(frames[0].gauss)
    out = []
    for f in frames:
        df = E.to_device(f, n_gauss=K)
        rnk = torch.empty(5 * f.n_sv, dtype=torch.float32, device="cuda")
        ind = torch.empty(5 * f.n_sv, dtype=torch.int32, device="cuda")
        st = plan.run_device(df, gm, rnk, ind, prm, stats=True)
        out.append(dict(rnk=rnk.cpu().numpy(), ind=ind.cpu().numpy(), gauss=E.gauss_from_device(gm), stats=st))
        E.update_priors(gm, K, 0.01, 1.0, 0.8, -1.0, True)
    torch.cuda.synchronize()
    plan.close()
    return out


def same_records(a, b):
    for name in L.GAUSS_DTYPE.names:
        np.testing.assert_array_equal(a[name], b[name], err_msg=name)


@pytest.mark.parametrize("form", ["float", "compact", "runs"])
def test_served_mix_is_bit_identical_to_alone(cuda_ok, form):
    from tgmm_b200.serve import Server
    prm = params()
    series = lineages()
    alone = [run_alone(fr, prm) for fr in series]
    with Server(params=prm, lanes=2, max_batch_frames=8) as srv:
        ids = [srv.open_lineage(fr[0].gauss) for fr in series]
        for t in range(N_FRAMES):  # interleaved arrivals of all lineages
            for li, fr in enumerate(series):
                srv.submit(ids[li], fr[t], tag=li * 100 + t, compact=form == "compact", runs=form == "runs")
        res = {r.tag: r for r in srv.drain()}
        st = srv.stats()
    assert len(res) == len(series) * N_FRAMES
    assert st["batches"] < len(series) * N_FRAMES  # frames of different lineages shared batches
    for li in range(len(series)):
        for t in range(N_FRAMES):
            r = res[li * 100 + t]
            assert r.status == L.TGMM_OK
            a = alone[li][t]
            np.testing.assert_array_equal(r.ind, a["ind"])
            np.testing.assert_array_equal(r.rnk, a["rnk"])
            same_records(r.gauss, a["gauss"])
            assert r.stats["iterations"] == a["stats"]["iterations"]
            assert r.stats["ll"] == a["stats"]["ll"]


def test_admission_against_a_small_budget(cuda_ok):
    from tgmm_b200.serve import Server
    prm = params()
    series = lineages()[:3]
    alone = [run_alone(fr, prm) for fr in series]
    lineage_bytes = sum(((fr[0].n_gauss * 288 + 255) // 256) * 256 for fr in series)
    biggest = max(16 * f.n_vox + 60 * f.n_sv + 2048 for fr in series for f in fr)
    budget = lineage_bytes + int(1.5 * biggest)  # room for about one frame at a time
    with Server(params=prm, lanes=2, hbm_budget=budget) as srv:
        ids = [srv.open_lineage(fr[0].gauss) for fr in series]
        for t in range(N_FRAMES):
            for li, fr in enumerate(series):
                srv.submit(ids[li], fr[t], tag=li * 100 + t)
        res = {r.tag: r for r in srv.drain()}
        st = srv.stats()
    assert st["hbm_peak"] <= st["hbm_budget"]
    for li in range(len(series)):
        for t in range(N_FRAMES):
            r = res[li * 100 + t]
            assert r.status == L.TGMM_OK
            np.testing.assert_array_equal(r.rnk, alone[li][t]["rnk"])
            same_records(r.gauss, alone[li][t]["gauss"])


def test_frames_that_can_never_run_are_answered(cuda_ok):
    from tgmm_b200.serve import Server
    fr = lineages()[0]
    K = fr[0].n_gauss
    small = ((K * 288 + 255) // 256) * 256 + 4096
    with Server(params=params(), lanes=1, hbm_budget=small, max_batch_sv=50) as srv:
        lid = srv.open_lineage(fr[0].gauss)
        srv.submit(lid, fr[0], tag=1)            # needs more than the budget holds
        srv.submit(lid + 7, fr[0], tag=2)        # unknown lineage
        res = {r.tag: r for r in srv.drain()}
    assert res[1].status == L.TGMM_ERR_ADMISSION
    assert res[2].status == L.TGMM_ERR_INVALID_ARG


def test_two_frame_lineage_against_the_oracle(cuda_ok):
    from oracle import oracle as O
    from tgmm_b200.serve import Server
    fr = lineages()[1][:2]
    prm = params(tol=-1.0)
    with Server(params=prm, lanes=1) as srv:
        lid = srv.open_lineage(fr[0].gauss)
        for t, f in enumerate(fr):
            srv.submit(lid, f, tag=t)
        res = {r.tag: r for r in srv.drain()}
    g = fr[0].gauss.copy()
    for t, f in enumerate(fr):
        o = O.em_run(f.query, f.img, f.centroids, f.label_ptr, g, O.params(max_iter=20, tol=-1.0))
        r = res[t]
        np.testing.assert_array_equal(r.ind, o["ind"])
        assert np.max(np.abs(r.rnk - o["rnk"])) <= 1e-5
        alive = o["gauss"]["m_o"][:, 0] > -1e31
        assert np.max(np.abs(r.gauss["m_k"][alive] - o["gauss"]["m_k"][alive])) <= 1e-3
        ws = np.max(np.abs(o["gauss"]["W_k"][alive]), axis=1, keepdims=True)
        assert np.max(np.abs(r.gauss["W_k"][alive] - o["gauss"]["W_k"][alive]) / ws) <= 1e-4
        g = o["gauss"].copy()
        atot = float(g["alpha_k"].sum())
        O.lib().or_update_priors(g.ctypes.data, g.shape[0], 0.01, 1.0, 0.8, atot)


def test_read_lineage_returns_the_next_prior(cuda_ok):
    import torch
    from tgmm_b200 import engine as E
    from tgmm_b200.serve import Server
    fr = lineages()[0][:1]
    prm = params()
    with Server(params=prm, lanes=1) as srv:
        lid = srv.open_lineage(fr[0].gauss)
        srv.submit(lid, fr[0], tag=0)
        post = srv.drain()[0].gauss
        prior = srv.read_lineage(lid)
    gm = E.gauss_to_device(post)
    E.update_priors(gm, post.shape[0], 0.01, 1.0, 0.8, -1.0, True)
    torch.cuda.synchronize()
    same_records(prior, E.gauss_from_device(gm))


def test_outputs_in_page_locked_memory_are_written_in_place(cuda_ok):
    import torch
    from tgmm_b200.serve import Server
    prm = params()
    series = lineages()[:2]
    alone = [run_alone(fr, prm) for fr in series]

    def pinned_out(S, K):
        return (torch.empty(5 * S).pin_memory().numpy(), torch.empty(5 * S, dtype=torch.int32).pin_memory().numpy(),
                torch.empty(K * 288, dtype=torch.uint8).pin_memory().numpy().view(L.GAUSS_DTYPE))
    with Server(params=prm, lanes=2) as srv:
        ids = [srv.open_lineage(fr[0].gauss) for fr in series]
        outs = {}
        for t in range(N_FRAMES):
            for li, fr in enumerate(series):
                outs[li * 100 + t] = pinned_out(fr[t].n_sv, fr[0].n_gauss)
                srv.submit(ids[li], fr[t], tag=li * 100 + t, out=outs[li * 100 + t])
        res = {r.tag: r for r in srv.drain()}
    for li in range(len(series)):
        for t in range(N_FRAMES):
            r, o = res[li * 100 + t], outs[li * 100 + t]
            assert r.status == L.TGMM_OK
            assert r.rnk.ctypes.data == o[0].ctypes.data
            np.testing.assert_array_equal(o[0], alone[li][t]["rnk"])
            np.testing.assert_array_equal(o[1], alone[li][t]["ind"])
            same_records(o[2], alone[li][t]["gauss"])


def test_frame_expand_gives_the_host_arrays(cuda_ok):
    """tgmm_frame_expand (the compact 6-byte voxel upload on the plain path) rebuilds the
    frame's float coordinates and intensities bit for bit."""
    import torch
    from tgmm_b200 import engine as E
    for name in ("c1", "big"):
        f = F.frame(name)
        lin, raw, dims, off, den = f.compact()
        q = torch.full((3 * f.n_vox,), float("nan"), device="cuda")
        im = torch.full((f.n_vox,), float("nan"), device="cuda")
        E.expand_frame(torch.from_numpy(lin.view(np.int32)).cuda(), torch.from_numpy(raw.view(np.int16)).cuda(),
                       dims, off, den, q, im)
        np.testing.assert_array_equal(q.cpu().numpy().view(np.uint32), f.query.view(np.uint32))
        np.testing.assert_array_equal(im.cpu().numpy().view(np.uint32), f.img.view(np.uint32))


def _expand_runs(f, rp, rs, rl, raw, dims, off, den):
    import torch
    from tgmm_b200 import engine as E
    q = torch.full((3 * f.n_vox,), float("nan"), device="cuda")
    im = torch.full((f.n_vox,), float("nan"), device="cuda")
    E.expand_runs(torch.from_numpy(rp).cuda(), torch.from_numpy(rs.view(np.int32)).cuda(),
                  torch.from_numpy(rl.view(np.int16)).cuda(), torch.from_numpy(raw.view(np.int16)).cuda(),
                  torch.from_numpy(np.ascontiguousarray(f.label_ptr)).cuda(), dims, off, den, q, im)
    return q.cpu().numpy(), im.cpu().numpy()


@pytest.mark.parametrize("name", ["tiny", "c1", "big", "split"])
def test_frame_expand_runs_gives_the_host_arrays(cuda_ok, name):
    """tgmm_frame_expand_runs (runs of consecutive linear indices, about 3 bytes a voxel) rebuilds
    the frame's float coordinates and intensities bit for bit; supervoxels with more than 32
    runs ("big") and many small supervoxels ("split") included."""
    f = F.frame(name)
    rp, rs, rl, raw, dims, off, den = f.runs()
    assert rs.shape[0] < f.n_vox
    q, im = _expand_runs(f, rp, rs, rl, raw, dims, off, den)
    np.testing.assert_array_equal(q.view(np.uint32), f.query.view(np.uint32))
    np.testing.assert_array_equal(im.view(np.uint32), f.img.view(np.uint32))


def test_frame_expand_runs_with_runs_cut_short(cuda_ok):
    """The same frame with every run cut to at most 3 voxels (many runs per supervoxel, several
    groups of 32 per warp) gives the same arrays."""
    f = F.frame("c1")
    lin, raw, dims, off, den = f.compact()
    rp, rs, rl = synth.runs_of(lin, f.label_ptr, max_len=3)
    q, im = _expand_runs(f, rp, rs, rl, raw, dims, off, den)
    np.testing.assert_array_equal(q.view(np.uint32), f.query.view(np.uint32))
    np.testing.assert_array_equal(im.view(np.uint32), f.img.view(np.uint32))


def test_frame_expand_runs_never_writes_outside_a_supervoxel(cuda_ok):
    """A run table that claims more voxels than a supervoxel holds writes nothing past the
    supervoxel's range: the next supervoxel's voxels and the array ends keep their values."""
    import torch
    from tgmm_b200 import engine as E
    lp = np.array([0, 4, 10], np.int64)
    rp = np.array([0, 1, 2], np.int32)
    rs = np.array([100, 500], np.uint32)
    rl = np.array([9, 6], np.uint16)  # supervoxel 0 holds 4 voxels, the table says 9
    raw = np.arange(200, 210, dtype=np.uint16)
    q = torch.full((30,), -1.0, device="cuda")
    im = torch.full((10,), -1.0, device="cuda")
    E.expand_runs(torch.from_numpy(rp).cuda(), torch.from_numpy(rs.view(np.int32)).cuda(),
                  torch.from_numpy(rl.view(np.int16)).cuda(), torch.from_numpy(raw.view(np.int16)).cuda(),
                  torch.from_numpy(lp).cuda(), (64, 64, 8), 150.0, 100.0, q, im)
    x = q.cpu().numpy()[:10]
    np.testing.assert_array_equal(x[:4], [36, 37, 38, 39])   # 100..103 in rows of 64
    np.testing.assert_array_equal(x[4:], [52, 53, 54, 55, 56, 57])  # supervoxel 1 from 500
