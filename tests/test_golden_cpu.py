"""Pins the CPU oracle to the reference's own outputs (tests/golden, produced by the
reference's GPU EM compiled from its sources; see tests/golden/make_golden.py).

* REF32 mode restates the reference's FP32 arithmetic and reduction order: candidate
  arrays identical (same replacement rule and slot order), responsibilities and means
  identical, precision matrices equal to 1e-6 relative.
* FP64 mode is the oracle the CUDA path is held to: the same kNN sets, survivors and
  supervoxel assignments as the reference; the remaining difference is the reference's
  FP32 accumulation (responsibilities <= 1e-4, means <= 1e-3 voxel, precision matrices
  <= 5e-3 relative)."""
import os

import numpy as np
import pytest

import _fixtures as F
import _golden as G
from oracle import oracle as O


@pytest.mark.parametrize("name", G.CASES)
def test_fixture_inputs_are_the_seeded_workload(name):
    z = G.load(name)
    assert str(z["input_sha256"]) == G.input_digest(F.frame(name)), \
        "the workload generator changed: regenerate tests/golden with make_golden.py on a GPU"


@pytest.mark.parametrize("name", G.CASES)
def test_reference_knn_slot_order(name):
    z, f = G.load(name), F.frame(name)
    ref_xyz = np.ascontiguousarray(f.gauss["m_k"].astype(np.float32)).reshape(-1)
    np.testing.assert_array_equal(O.knn(f.centroids, ref_xyz, reference_rule=True), z["knn_ind"])
    S = f.n_sv
    np.testing.assert_array_equal(np.sort(O.knn(f.centroids, ref_xyz).reshape(5, S), 0),
                                  np.sort(z["knn_ind"].reshape(5, S), 0))


@pytest.mark.parametrize("it", G.ITERS)
@pytest.mark.parametrize("name", G.CASES)
def test_ref32_oracle_reproduces_reference(name, it):
    z, f = G.load(name), F.frame(name)
    o = O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss,
                 O.params(max_iter=it, tol=-1.0, mode=O.MODE_REF32))
    G.compare_with_reference(z, it, o, f.n_sv, rnk_tol=1e-6, m_tol=1e-6, w_rtol=1e-6, same_slot_order=True)


@pytest.mark.parametrize("it", G.ITERS)
@pytest.mark.parametrize("name", G.CASES)
def test_fp64_oracle_agrees_with_reference(name, it):
    z, f = G.load(name), F.frame(name)
    o = O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss,
                 O.params(max_iter=it, tol=-1.0, mode=O.MODE_FP64))
    G.compare_with_reference(z, it, o, f.n_sv, rnk_tol=1e-4, m_tol=1e-3, w_rtol=5e-3, same_slot_order=False)


def _local_golden():
    with np.load(os.path.join(G.GOLDEN, "local_ll.npz")) as z:
        return {k: z[k] for k in z.files}


LOCAL_CASES = ["c1", "hard", "big"]


@pytest.mark.parametrize("name", LOCAL_CASES)
def test_local_likelihood_oracle_reproduces_reference(name):
    """The oracle's local log-likelihood against the reference's own calculateLocalLikelihood
    (tests/golden/local_ll.npz, written by make_local_golden.py after the reference's own EM):
    the float-sum mode to 1e-6 relative, the FP64 mode to the reference's float error."""
    z, f = _local_golden(), F.frame(name)
    assert str(z[f"{name}_input_sha256"]) == G.input_digest(f)
    ptr, idx = z[f"{name}_list_ptr"], z[f"{name}_list_idx"]
    lists = [list(idx[ptr[i]:ptr[i + 1]]) for i in range(ptr.shape[0] - 1)]
    args = (f.query, f.img, f.label_ptr, z[f"{name}_ind"], z[f"{name}_gauss"], lists)
    np.testing.assert_allclose(O.local_likelihood(*args, mode=O.MODE_REF32), z[f"{name}_ll"], rtol=1e-6)
    np.testing.assert_allclose(O.local_likelihood(*args), z[f"{name}_ll"], rtol=2e-5)
