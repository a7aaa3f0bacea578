"""The exact fallback branches and the bounded wait of the EM kernels, each forced on a
small frame and checked against the FP64 oracle (or, for the wait, checked to report and
to leave the plan usable).

- "split" (every supervoxel cut into ~12-voxel pieces): each Gaussian is a candidate of far
  more than the 32 (slot, supervoxel) pairs its M-step bucket holds, and takes more than 32
  supervoxels with rnk > 0.5, so its M-step sums and its supervoxelIdx list come from the
  ordered block-wide scans (TGMM_FLAG_BUCKET_OVERFLOW, TGMM_FLAG_ASSIGN_OVERFLOW).  The
  reference keeps the first 16 assignments in (slot, supervoxel) order
  (GMEMupdateCUDA.cu:4310-4350); so does the oracle.
- "crowded" (40 near-copies of one Gaussian): more centres in one kNN grid cell than the
  cell holds, so the frame's kNN scans every Gaussian (TGMM_FLAG_CELL_OVERFLOW).
- A wait limit of 1 ns on the voxel passes' tile copies: the copies cannot land in time, the
  call returns TGMM_ERR_DEVICE_FLAG with TGMM_FLAG_STAGE_TIMEOUT, and the next call on the
  same plan, with the default limit, matches a fresh plan bit for bit.
"""
import numpy as np
import pytest

import _fixtures as F
from _parity import compare
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run(name, iters):
    import torch
    from tgmm_b200 import engine as E
    f = F.frame(name)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    out = plan.run_host(E.to_device(f), f.gauss, F.params(iters))
    plan.close()
    torch.cuda.synchronize()
    return out


def _oracle(name, iters):
    f = F.frame(name)
    return O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, O.params(max_iter=iters, tol=-1.0))


def test_bucket_and_assignment_overflow_take_the_ordered_scans(cuda_ok):
    from tgmm_b200 import _lib as L
    g = _run("split", 20)
    assert g["device_flags"] & L.TGMM_FLAG_BUCKET_OVERFLOW
    assert g["device_flags"] & L.TGMM_FLAG_ASSIGN_OVERFLOW
    o = _oracle("split", 20)
    assert o["gauss"]["supervoxelNum"].max() == 16  # the reference's cap is reached
    compare(g, o)


def test_cell_overflow_scans_every_gaussian(cuda_ok):
    from tgmm_b200 import _lib as L
    g = _run("crowded", 20)
    assert g["device_flags"] & L.TGMM_FLAG_CELL_OVERFLOW
    compare(g, _oracle("crowded", 20))


def test_stage_wait_limit_reports_and_the_plan_recovers(cuda_ok):
    import torch
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame("c1")
    df = E.to_device(f)
    prm = F.params(5)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    plan.set_stage_wait(1)
    rc, st = plan.run_host_status(df, f.gauss, prm)
    torch.cuda.synchronize()
    assert rc == L.TGMM_ERR_DEVICE_FLAG
    assert st["device_flags"] & L.TGMM_FLAG_STAGE_TIMEOUT
    assert b"wait limit" in L.gmem().tgmm_last_error()
    plan.set_stage_wait(1_000_000_000)
    again = plan.run_host(df, f.gauss, prm)
    plan.close()
    fresh = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    want = fresh.run_host(df, f.gauss, prm)
    fresh.close()
    assert again["device_flags"] == 0
    assert L.records_equal(again["gauss"], want["gauss"])
    np.testing.assert_array_equal(again["rnk"], want["rnk"])
    np.testing.assert_array_equal(again["ind"], want["ind"])
    compare(again, _oracle("c1", 5))
