"""The allocation-free kNN entry point (tgmm_knn_noalloc).

Some callers of this library cannot allocate device memory: their device memory belongs
to another allocator (a framework's caching pool, a host application's fixed arena), or
they run where an allocation's latency or failure is not acceptable.  tgmm_knn_noalloc
serves them from a fixed scratch array compiled into the library.  This test calls it
through the C ABI twice in a row and checks each result against the allocating entry
point tgmm_knn (exact: kNN indices are integers), and that sizes beyond the scratch are
refused.  It lives in its own file so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

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


def test_knn_noalloc_matches_allocating_knn_twice(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    rng = np.random.default_rng(42)
    cases = [(3000, 2500), (20000, 20000)]  # two calls in a row, different sizes
    for nq, nref in cases:
        q = torch.from_numpy(rng.uniform(0, 300, size=3 * nq).astype(np.float32)).cuda()
        r = torch.from_numpy(rng.uniform(0, 300, size=3 * nref).astype(np.float32)).cuda()
        rc, got = _call_noalloc(q, r)
        assert rc == L.TGMM_OK, L.gmem().tgmm_last_error()
        want = E.knn(q, r)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())


def test_knn_noalloc_refuses_sizes_beyond_its_scratch(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    q = torch.zeros(3 * 4, dtype=torch.float32, device="cuda")
    r = torch.zeros(3 * 65536, dtype=torch.float32, device="cuda")
    rc, _ = _call_noalloc(q, r)
    assert rc == L.TGMM_ERR_BAD_SIZE
    assert b"65535" in L.gmem().tgmm_last_error()
