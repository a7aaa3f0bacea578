"""The tracking graph's supervoxel kNN (tgmm_knn_k, and the reference-named knnCUDA_ over it):
the k nearest (k <= 11) with their squared scaled distances, bit for bit the oracle's
(distance, index) order, and the same neighbour sets and distances as the reference's own
kernel compiled from its sources."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
SCALE = (1.0, 1.0, 2.0)


def gpu_knn_k(q, r, k):
    import torch
    from tgmm_b200 import _lib as L
    nq, nref = q.size // 3, r.size // 3
    qd, rd = torch.from_numpy(q).cuda(), torch.from_numpy(r).cuda()
    ind = torch.empty(k * max(nq, 1), dtype=torch.int32, device="cuda")
    dist = torch.empty(k * max(nq, 1), dtype=torch.float32, device="cuda")
    sc = (C.c_float * 3)(*SCALE)
    rc = L.gmem().tgmm_knn_k(qd.data_ptr(), nq, rd.data_ptr(), nref, k, sc, ind.data_ptr(), dist.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
    assert rc == L.TGMM_OK
    torch.cuda.synchronize()
    return ind.cpu().numpy()[:k * nq], dist.cpu().numpy()[:k * nq]


def cases():
    rng = np.random.default_rng(11)
    for nq, nref in [(1, 1), (37, 5), (1000, 300), (5000, 4000), (20000, 20000), (50, 3)]:
        q = rng.uniform(0, 200, size=(3, nq)).astype(np.float32)
        r = rng.uniform(0, 200, size=(3, nref)).astype(np.float32)
        if nref > 20:  # exact duplicates and lattice points: distance ties
            r[:, 5:10] = r[:, :1]
            r[:, 10:20] = np.round(r[:, 10:20])
            q[:, :10] = np.round(q[:, :10])
        yield q.reshape(-1), r.reshape(-1)


@pytest.mark.parametrize("k", [1, 3, 5, 8, 11])
def test_knn_k_is_the_oracles(cuda_ok, k):
    for q, r in cases():
        gi, gd = gpu_knn_k(q, r, k)
        oi, od = O.knn_topk(q, r, k, SCALE)
        np.testing.assert_array_equal(gi, oi)
        np.testing.assert_array_equal(gd, od)


def test_reference_named_entry_point_with_host_arrays(cuda_ok):
    from tgmm_b200 import _lib as L
    f = L.gmem()["_Z8knnCUDA_PiPfS0_S0_xiiS0_i"]
    f.restype = C.c_int
    vp = C.c_void_p
    f.argtypes = [vp, vp, vp, vp, C.c_longlong, C.c_int, C.c_int, vp, C.c_int]
    q, r = next(x for i, x in enumerate(cases()) if i == 2)
    k = 11
    nq, nref = q.size // 3, r.size // 3
    ind, dist = np.zeros(k * nq, np.int32), np.zeros(k * nq, np.float32)
    sc = np.asarray(SCALE, np.float32)
    assert f(ind.ctypes.data, dist.ctypes.data, q.ctypes.data, r.ctypes.data, nq, nref, k, sc.ctypes.data, 0) == 0
    oi, od = O.knn_topk(q, r, k, SCALE)
    np.testing.assert_array_equal(ind, oi)
    np.testing.assert_array_equal(dist, od)


@pytest.mark.parametrize("k", [2, 5, 11])
def test_knn_k_matches_the_reference_kernel(cuda_ok, k):
    """Against the reference's own kernel (<= 1024 queries: one full block, see the harness):
    its slots come in replacement order, so both sides are compared as sorted sets; the
    points are random, without ties."""
    if not O.ref_f3_available():
        pytest.skip("oracle/_ref/libtgmm_ref_f3.so not built (oracle/build_ref.sh needs the reference sources)")
    rng = np.random.default_rng(5)
    for nq, nref in [(1024, 3000), (300, 40), (1000, 1000)]:
        q = rng.uniform(0, 300, size=(3, nq)).astype(np.float32).reshape(-1)
        r = rng.uniform(0, 300, size=(3, nref)).astype(np.float32).reshape(-1)
        ri, rd = O.ref_knn_k(q, r, k, SCALE)
        gi, gd = gpu_knn_k(q, r, k)
        ri, rd, gi, gd = (a.reshape(k, nq) for a in (ri, rd, gi, gd))
        order = np.lexsort((ri, rd), axis=0)
        np.testing.assert_array_equal(np.take_along_axis(ri, order, 0), gi)
        np.testing.assert_array_equal(np.take_along_axis(rd, order, 0), gd)
