"""Frame preparation on the device (tgmm_frame_build): from the raw 16-bit image and the
segmentation's label volume to the EM's input arrays, bit for bit the oracle's restatement of
the tracking program's host build (itself pinned to the reference's own trimming and
statistics code), with its error behaviour, and an EM run on the built frame identical to one
on the oracle's arrays."""
import ctypes as C

import numpy as np
import pytest

import _fixtures as F
import _volumes as V
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=1),
    dict(seed=2, conn=26),
    dict(seed=3, max_size=60),
    dict(seed=4, max_pct=0.15, conn=8),
    dict(seed=5, conn=4, min_size=20),
    dict(seed=6, conn=74, max_size=200),
    dict(seed=9, dims=(160, 144, 40), n_nuclei=120),
    dict(seed=10, dims=(512, 512, 64), n_nuclei=1500),  # 16.8M voxels
    dict(seed=15, big=True, dims=(160, 144, 40), n_nuclei=80),  # a box beyond the shared-memory flood
]


def _params(case):
    c = dict(max_size=3000, max_pct=0.4, conn=6, min_size=50)
    c.update({k: case[k] for k in c if k in case})
    return c


def _volume(case):
    kw = {k: case[k] for k in ("dims", "n_nuclei", "big") if k in case}
    return V.make(seed=case["seed"], **kw)


def device_build(raw, lab, n, c, max_vox=None, max_sv=None):
    import torch
    from tgmm_b200 import engine as E
    Z, Y, X = raw.shape
    b = E.FrameBuilder((X, Y, Z), n, max_nuclei_size=c["max_size"], max_percentile=c["max_pct"], conn3d=c["conn"],
                       min_nuclei_size=c["min_size"])
    rd = torch.from_numpy(raw.reshape(-1).view(np.int16)).cuda()
    ld = torch.from_numpy(lab.reshape(-1).view(np.int32)).cuda()
    f, thr = b.build(rd, ld)
    torch.cuda.synchronize()
    return f, thr


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_device_build_is_the_oracles(cuda_ok, case):
    c = _params(case)
    raw, lab, n = _volume(case)
    rc, o = O.frame_build(raw, lab, n, O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"]))
    assert rc == 0
    f, thr = device_build(raw, lab, n, c)
    assert (f.n_vox, f.n_sv) == (o["n_vox"], o["n_sv"])
    np.testing.assert_array_equal(f.label_ptr.cpu().numpy(), o["lptr"])
    np.testing.assert_array_equal(thr, o["thr"])
    np.testing.assert_array_equal(f.query.cpu().numpy(), o["query"])
    np.testing.assert_array_equal(f.img.cpu().numpy().view(np.uint32), o["img"].view(np.uint32))
    np.testing.assert_array_equal(f.centroids.cpu().numpy().view(np.uint32), o["cent"].view(np.uint32))


def test_device_build_is_repeatable(cuda_ok):
    raw, lab, n = V.make(seed=12)
    c = _params({})
    a, ta = device_build(raw, lab, n, c)
    qa, ia = a.query.cpu().numpy().copy(), a.img.cpu().numpy().copy()
    b, tb = device_build(raw, lab, n, c)
    np.testing.assert_array_equal(qa, b.query.cpu().numpy())
    np.testing.assert_array_equal(ia, b.img.cpu().numpy())
    np.testing.assert_array_equal(ta, tb)


def _raw_call(raw, lab, n, c, max_vox, max_sv):
    import torch
    from tgmm_b200 import _lib as L
    Z, Y, X = raw.shape
    lib = L.gmem()
    dims = (C.c_int32 * 3)(X, Y, Z)
    p = L.TgmmFrameBuildParams(c["max_size"], c["max_pct"], c["conn"], c["min_size"])
    ws = torch.empty(lib.tgmm_frame_build_bytes(dims, n), dtype=torch.uint8, device="cuda")
    rd = torch.from_numpy(raw.reshape(-1).view(np.int16)).cuda()
    ld = torch.from_numpy(lab.reshape(-1).view(np.int32)).cuda()
    q = torch.empty(3 * max(max_vox, 1), dtype=torch.float32, device="cuda")
    im = torch.empty(max(max_vox, 1), dtype=torch.float32, device="cuda")
    ce = torch.empty(3 * max(max_sv, 1), dtype=torch.float32, device="cuda")
    lp = torch.empty(max_sv + 1, dtype=torch.int64, device="cuda")
    nv, ns = C.c_int64(-1), C.c_int32(-1)
    rc = lib.tgmm_frame_build(rd.data_ptr(), ld.data_ptr(), dims, n, C.byref(p), ws.data_ptr(), ws.numel(),
                              q.data_ptr(), im.data_ptr(), ce.data_ptr(), lp.data_ptr(), None, max_vox, max_sv,
                              C.byref(nv), C.byref(ns), torch.cuda.current_stream().cuda_stream)
    return rc, nv.value, ns.value, lib.tgmm_last_error()


def test_device_build_errors(cuda_ok):
    from tgmm_b200 import _lib as L
    raw, lab, n = V.make(seed=13)
    c = _params({})
    rc0, o = O.frame_build(raw, lab, n)
    nvol = raw.size
    # outputs too small: nothing written, the sizes reported
    rc, nv, ns, _ = _raw_call(raw, lab, n, c, o["n_vox"] - 1, n)
    assert rc == L.TGMM_ERR_BAD_SIZE and (nv, ns) == (o["n_vox"], o["n_sv"])
    rc, nv, ns, _ = _raw_call(raw, lab, n, c, nvol, o["n_sv"] - 1)
    assert rc == L.TGMM_ERR_BAD_SIZE and ns == o["n_sv"]
    # every supervoxel below the minimum size: the reference's exit(5)
    rc, nv, ns, msg = _raw_call(raw, lab, n, dict(c, min_size=10 ** 6), nvol, n)
    assert rc == L.TGMM_ERR_NO_SUPERVOXEL and b"erased" in msg
    # a label above n_labels
    bad = lab.copy()
    bad[1, 2, 3] = n + 5
    rc, nv, ns, msg = _raw_call(raw, bad, n, c, nvol, n)
    assert rc == L.TGMM_ERR_INVALID_ARG and b"label" in msg
    # the library is usable afterwards
    rc, nv, ns, _ = _raw_call(raw, lab, n, c, nvol, n)
    assert rc == L.TGMM_OK and (nv, ns) == (o["n_vox"], o["n_sv"])


def test_em_on_the_built_frame_is_the_em_on_the_oracles_arrays(cuda_ok):
    """The built arrays feed the EM directly; the run equals one on the same arrays uploaded."""
    import torch
    from tgmm_b200 import engine as E
    raw, lab, n = V.make(seed=14, dims=(128, 112, 32), n_nuclei=60)
    c = _params({})
    rc, o = O.frame_build(raw, lab, n)
    assert rc == 0
    f, _ = device_build(raw, lab, n, c)
    S = o["n_sv"]
    # the inputs first: the built arrays are the oracle's bits
    np.testing.assert_array_equal(f.query.cpu().numpy(), o["query"])
    np.testing.assert_array_equal(f.img.cpu().numpy().view(np.uint32), o["img"].view(np.uint32))
    np.testing.assert_array_equal(f.centroids.cpu().numpy().view(np.uint32), o["cent"].view(np.uint32))
    np.testing.assert_array_equal(f.label_ptr.cpu().numpy(), o["lptr"])
    g = np.repeat(F.frame("hard").gauss[:1], S)
    cent = o["cent"].reshape(3, S).T.astype(np.float64)
    g["m_k"] = cent
    g["m_o"] = cent
    f.n_gauss = S
    up = E.DeviceFrame(torch.from_numpy(o["query"]).cuda(), torch.from_numpy(o["img"]).cuda(),
                       torch.from_numpy(o["cent"]).cuda(), torch.from_numpy(o["lptr"]).cuda(), S)
    plan = E.Plan(o["n_vox"], S, S)
    prm = F.params(iters=10)
    a = plan.run_host(f, g, prm)
    b = plan.run_host(up, g, prm)
    np.testing.assert_array_equal(a["rnk"], b["rnk"])
    np.testing.assert_array_equal(a["ind"], b["ind"])
    # equal inputs give equal bytes: every field of every Gaussian record, the rows that
    # differ named in the message
    for name in a["gauss"].dtype.names:
        x, y = np.ascontiguousarray(a["gauss"][name]), np.ascontiguousarray(b["gauss"][name])
        rows = np.flatnonzero((x.view(np.uint8).reshape(x.shape[0], -1) !=
                               y.view(np.uint8).reshape(y.shape[0], -1)).any(axis=1))
        assert rows.size == 0, (name, rows[:10].tolist(), x[rows[:3]], y[rows[:3]])


def _lists(raw, lab, n):
    """The segmentation as the tracking program holds it: per supervoxel its voxels' linear
    indices, ascending (PixelIdxList), with their raw values."""
    ptr, lin = O.supervoxel_lists(lab, n)
    return ptr.astype(np.int64), lin.astype(np.uint32), raw.reshape(-1)[lin.astype(np.int64)].astype(np.uint16)


def list_build(raw, lab, n, c):
    import torch
    from tgmm_b200 import engine as E
    Z, Y, X = raw.shape
    b = E.FrameBuilder((X, Y, Z), n, max_nuclei_size=c["max_size"], max_percentile=c["max_pct"], conn3d=c["conn"],
                       min_nuclei_size=c["min_size"])
    ptr, lin, val = _lists(raw, lab, n)
    f, thr = b.build_lists(torch.from_numpy(lin.view(np.int32)).cuda(), torch.from_numpy(val.view(np.int16)).cuda(),
                           torch.from_numpy(ptr).cuda())
    torch.cuda.synchronize()
    return f, thr


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_list_build_is_the_oracles(cuda_ok, case):
    """tgmm_frame_build_lists (the segmentation as per-supervoxel pixel lists, no volume on the
    device) gives the oracle's arrays bit for bit, as the volume form does; the last volume
    holds a supervoxel whose box exceeds the shared-memory flood (binary search in its list)."""
    c = _params(case)
    raw, lab, n = _volume(case)
    rc, o = O.frame_build(raw, lab, n, O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"]))
    assert rc == 0
    f, thr = list_build(raw, lab, n, c)
    assert (f.n_vox, f.n_sv) == (o["n_vox"], o["n_sv"])
    np.testing.assert_array_equal(f.query.cpu().numpy().view(np.uint32), o["query"].view(np.uint32))
    np.testing.assert_array_equal(f.img.cpu().numpy().view(np.uint32), o["img"].view(np.uint32))
    np.testing.assert_array_equal(f.centroids.cpu().numpy().view(np.uint32), o["cent"].view(np.uint32))
    np.testing.assert_array_equal(f.label_ptr.cpu().numpy(), o["lptr"])
    np.testing.assert_array_equal(thr, o["thr"])


def test_list_build_refuses_lists_out_of_order(cuda_ok):
    """A list that is not ascending, or leaves the volume, is refused (TGMM_ERR_DEVICE_FLAG),
    and the builder works afterwards."""
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    raw, lab, n = _volume(dict(seed=1))
    Z, Y, X = raw.shape
    ptr, lin, val = _lists(raw, lab, n)
    b = E.FrameBuilder((X, Y, Z), n)
    for bad in ("swap", "outside"):
        l2 = lin.copy()
        a = int(ptr[3])
        if bad == "swap":
            l2[a], l2[a + 1] = l2[a + 1], l2[a]
        else:
            l2[a] = X * Y * Z + 5
        with pytest.raises(L.TgmmError) as ei:
            b.build_lists(torch.from_numpy(l2.view(np.int32)).cuda(), torch.from_numpy(val.view(np.int16)).cuda(),
                          torch.from_numpy(ptr).cuda())
        assert ei.value.code == L.TGMM_ERR_DEVICE_FLAG
    f, _ = b.build_lists(torch.from_numpy(lin.view(np.int32)).cuda(), torch.from_numpy(val.view(np.int16)).cuda(),
                         torch.from_numpy(ptr).cuda())
    rc, o = O.frame_build(raw, lab, n)
    np.testing.assert_array_equal(f.img.cpu().numpy().view(np.uint32), o["img"].view(np.uint32))
