"""Pins the CPU oracle to the reference itself: the reference's GPU path, compiled from
its own sources for sm_100a (oracle/_ref), runs the same seeded inputs, and the oracle's
REF32 mode (the reference's FP32 arithmetic and reduction order) must agree with it.
Only frames with at most 1024 supervoxels are run on the reference: its kNN kernel
returns early for surplus threads and then calls __syncthreads(), which is only
well-defined when no thread of the block returns early."""
import numpy as np
import pytest

import _fixtures as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = ["tiny", "small", "c1", "hard"]


def needs_ref():
    if not O.ref_available():
        pytest.skip("oracle/_ref/libtgmm_ref.so not built (oracle/build_ref.sh needs the reference sources)")


def canon_sets(ind, S):
    return np.sort(ind.reshape(5, S), axis=0)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("iters", [1, 20])
def test_reference_matches_oracle_ref32(cuda_ok, name, iters):
    needs_ref()
    f = F.frame(name)
    assert f.n_sv <= 1024
    r = O.ref_em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, max_iter=iters, tol=-1.0)
    o = O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss,
                 O.params(max_iter=iters, tol=-1.0, mode=O.MODE_REF32))
    # the same replacement rule and slot order -> identical candidate arrays
    np.testing.assert_array_equal(r["ind"], o["ind"])
    assert np.max(np.abs(r["rnk"] - o["rnk"])) <= 1e-4
    rg, og = r["gauss"], o["gauss"]
    alive = og["m_o"][:, 0] > -1e31
    np.testing.assert_array_equal(rg["m_o"][:, 0] > -1e31, alive)
    np.testing.assert_array_equal(rg["supervoxelNum"], og["supervoxelNum"])
    assert np.max(np.abs(rg["m_k"][alive] - og["m_k"][alive])) <= 1e-3
    ws = np.max(np.abs(og["W_k"][alive]), axis=1, keepdims=True)
    assert np.max(np.abs(rg["W_k"][alive] - og["W_k"][alive]) / ws) <= 1e-3


def test_padding_with_empty_supervoxels_leaves_the_reference_outputs_unchanged(cuda_ok):
    """The reference runs frames above 1024 supervoxels only padded to a multiple of 1024
    with empty supervoxels (its kNN kernel's early return before __syncthreads()).  On the C1
    frame (300 supervoxels, one block) the padded run (1024) gives the unpadded run's Gaussian
    records and the real supervoxels' candidates and responsibilities bit for bit."""
    needs_ref()
    f = F.frame("c1")
    S = f.n_sv
    a = O.ref_em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, max_iter=20, tol=-1.0)
    cp, lp = O.pad_supervoxels(f.centroids, f.label_ptr)
    assert lp.shape[0] - 1 == 1024
    b = O.ref_em_run(f.query, f.img, cp, lp, f.gauss, max_iter=20, tol=-1.0)
    Sp = lp.shape[0] - 1
    np.testing.assert_array_equal(b["ind"].reshape(5, Sp)[:, :S], a["ind"].reshape(5, S))
    np.testing.assert_array_equal(b["rnk"].reshape(5, Sp)[:, :S], a["rnk"].reshape(5, S))
    np.testing.assert_array_equal(b["rnk"].reshape(5, Sp)[:, S:], np.float32(0.2))  # 1/5 each
    for k in a["gauss"].dtype.names:
        np.testing.assert_array_equal(np.ascontiguousarray(b["gauss"][k]), np.ascontiguousarray(a["gauss"][k]),
                                      err_msg=k)


@pytest.mark.parametrize("name", CASES)
def test_reference_knn_sets_equal_canonical(cuda_ok, name):
    needs_ref()
    f = F.frame(name)
    ref_xyz = np.ascontiguousarray(f.gauss["m_k"].astype(np.float32)).reshape(-1)
    got = O.ref_knn(f.centroids, ref_xyz)
    S = f.n_sv
    np.testing.assert_array_equal(canon_sets(got, S), canon_sets(O.knn(f.centroids, ref_xyz), S))
    np.testing.assert_array_equal(got, O.knn(f.centroids, ref_xyz, reference_rule=True))


def test_gmm_xml_is_the_references(cuda_ok, tmp_path):
    """The library's GMM XML document is byte for byte the one the reference's own writer
    (compiled from its sources) makes for the same records: live, dead, fixed and twin
    Gaussians, before and after an EM run."""
    needs_ref()
    from tgmm_b200 import _lib as L
    from tgmm_b200 import engine as E
    f = F.frame("hard")
    g0 = np.ascontiguousarray(f.gauss)
    plan = E.Plan(f.n_vox, f.n_sv, f.n_gauss)
    try:
        g1 = plan.run_host(E.to_device(f), f.gauss, F.params(20, -1.0))["gauss"]
    finally:
        plan.close()
    for i, g in enumerate([g0, np.ascontiguousarray(g1)]):
        ours, ref = tmp_path / f"ours{i}.xml", tmp_path / f"ref{i}.xml"
        assert L.gmem().tgmm_write_gmm_xml(str(ours).encode(), g.ctypes.data, g.shape[0]) == L.TGMM_OK
        O.ref_write_gmm_xml(ref, g)
        assert ours.read_bytes() == ref.read_bytes()
