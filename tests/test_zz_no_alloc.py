"""The allocation-free kNN entry point (tgmm_knn_noalloc).

Some callers of this library cannot allocate device memory: their device memory belongs
to another allocator (a framework's caching pool, a host application's fixed arena), or
they run where an allocation's latency or failure is not acceptable.  tgmm_knn_noalloc
serves them from a fixed scratch array compiled into the library.  These tests call it
through the C ABI, two calls in a row, and check each result against the allocating entry
point tgmm_knn and against the oracle's brute-force kNN (exact: kNN indices are integers),
at its upper bound of 65535 reference points too; that sizes beyond the scratch are
refused; and that a call takes nothing from the device's memory pool, which the allocating
entry point does.  The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _call_noalloc(q, r, scale=(1.0, 1.0, 2.0)):
    import torch
    from tgmm_b200 import _lib as L
    nq = q.numel() // 3
    ind = torch.full((5 * nq,), -7, dtype=torch.int32, device=q.device)
    sc = (C.c_float * 3)(*scale)
    rc = L.gmem().tgmm_knn_noalloc(q.data_ptr(), nq, r.data_ptr(), r.numel() // 3, sc, ind.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    return rc, ind


def _points(rng, n, hi=300.0):
    p = rng.uniform(0, hi, size=3 * n).astype(np.float32)
    p[: 3 * min(n, 40)] = np.round(p[: 3 * min(n, 40)])  # lattice points: distance ties
    return p


def test_knn_noalloc_matches_allocating_knn_and_oracle_twice(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    rng = np.random.default_rng(42)
    # two calls in a row with different sizes (the second reuses the scratch the first
    # left), the last at the scratch's upper bound
    for nq, nref in [(3000, 2500), (20000, 20000), (4000, L_MAX_REF)]:
        qh, rh = _points(rng, nq), _points(rng, nref)
        q, r = torch.from_numpy(qh).cuda(), torch.from_numpy(rh).cuda()
        rc, got = _call_noalloc(q, r)
        assert rc == L.TGMM_OK, L.gmem().tgmm_last_error()
        want = E.knn(q, r)
        torch.cuda.synchronize()
        got = got.cpu().numpy()
        np.testing.assert_array_equal(got, want.cpu().numpy())
        np.testing.assert_array_equal(got, O.knn(qh, rh))


L_MAX_REF = 65535  # TGMM_KNN_NOALLOC_MAX_REF


def test_knn_noalloc_refuses_sizes_beyond_its_scratch(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    q = torch.zeros(3 * 4, dtype=torch.float32, device="cuda")
    r = torch.zeros(3 * (L_MAX_REF + 1), dtype=torch.float32, device="cuda")
    rc, _ = _call_noalloc(q, r)
    assert rc == L.TGMM_ERR_BAD_SIZE
    assert b"65535" in L.gmem().tgmm_last_error()


def _pool_high_after(fn):
    """The device's default memory pool (the one stream-ordered allocations draw on): its
    high-water mark of used bytes, reset just before fn runs, and its use before fn."""
    import torch
    from cuda.bindings import driver as drv
    torch.cuda.synchronize()
    err, dev = drv.cuCtxGetDevice()
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    used = drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    high = drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
    err, before = drv.cuMemPoolGetAttribute(pool, used)
    assert err == drv.CUresult.CUDA_SUCCESS
    (err,) = drv.cuMemPoolSetAttribute(pool, high, drv.cuuint64_t(0))  # resets the mark to the current use
    assert err == drv.CUresult.CUDA_SUCCESS
    fn()
    torch.cuda.synchronize()
    err, peak = drv.cuMemPoolGetAttribute(pool, high)
    assert err == drv.CUresult.CUDA_SUCCESS
    return int(before), int(peak)


def test_knn_noalloc_takes_no_device_memory(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    rng = np.random.default_rng(7)
    q = torch.from_numpy(_points(rng, 5000)).cuda()
    r = torch.from_numpy(_points(rng, 30000)).cuda()
    assert _call_noalloc(q, r)[0] == L.TGMM_OK  # the first call on the device looks the scratch up
    out = {}
    before, peak = _pool_high_after(lambda: out.setdefault("rc", _call_noalloc(q, r)[0]))
    assert out["rc"] == L.TGMM_OK
    assert peak <= before, (before, peak)
    # the check sees allocations: the allocating entry point's stream-ordered scratch shows
    before, peak = _pool_high_after(lambda: E.knn(q, r))
    assert peak > before
