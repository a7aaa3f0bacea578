"""The split proposal of the split round (GaussianMixtureModel::splitGaussian(GM, id),
GaussianMixtureModel.cpp:514-557, with updatePriorsAfterSplitProposal :912-922), on the CPU:
the library's host implementation (tgmm_split_proposal) equals the oracle's restatement, and
both equal the reference's own class compiled from its sources (oracle/_ref/libtgmm_ref_gmm.so,
built by oracle/build_ref.sh) to 1e-8, up to which half is which: the reference takes the
eigenvector's sign from its Eigen solver, these from the largest component.  The records are
the reference's own EM outputs (tests/golden), every live Gaussian."""
import ctypes as C

import numpy as np
import pytest

import _golden as G
from oracle import oracle as O
from tgmm_b200 import _lib as L

FIELDS = ("m_k", "W_k", "W_o", "m_o", "beta_o", "nu_o", "nu_k", "beta_k", "alpha_k", "alpha_o", "supervoxelNum")


def lib_split(rec, scale=(1.0, 1.0, 2.0)):
    g = np.ascontiguousarray(np.asarray(rec).reshape(1)).astype(L.GAUSS_DTYPE)
    a, b = g.copy(), g.copy()
    sc = (C.c_float * 3)(*scale)
    assert L.gmem().tgmm_split_proposal(g.ctypes.data, sc, a.ctypes.data, b.ctypes.data) == L.TGMM_OK
    return a[0], b[0]


def live_records():
    for name in ("c1", "hard"):
        g = G.load(name)["em20_gauss"]
        for k in range(g.shape[0]):
            if g["m_o"][k, 0] > -1e31:
                yield name, k, g[k]


def test_library_split_equals_the_oracle():
    n = 0
    for name, k, rec in live_records():
        for scale in ((1.0, 1.0, 2.0), (1.0, 1.0, 1.0)):
            la, lb = lib_split(rec, scale)
            oa, ob = O.split_proposal(rec, scale)
            for f in FIELDS:
                np.testing.assert_array_equal(la[f], oa[f], err_msg=f"{name} {k} {f}")
                np.testing.assert_array_equal(lb[f], ob[f], err_msg=f"{name} {k} {f}")
        n += 1
    assert n > 300


@pytest.mark.skipif(not O.ref_gmm_available(), reason="reference Gaussian class not built (oracle/build_ref.sh)")
def test_split_matches_the_reference_class():
    swapped = 0
    for name, k, rec in live_records():
        a, b = O.split_proposal(rec)
        ra, rb = O.ref_split_gaussian(rec)
        if np.max(np.abs(a["m_k"] - ra["m_k"])) > 1e-6:  # the halves trade places
            a, b = b, a
            swapped += 1
        for x, y in ((a, ra), (b, rb)):
            for f in ("m_k", "m_o"):
                assert np.max(np.abs(x[f] - y[f])) <= 1e-8, (name, k, f)
            for f in ("W_k", "W_o", "beta_o", "nu_o", "nu_k", "beta_k", "alpha_k", "alpha_o"):
                np.testing.assert_allclose(x[f], y[f], rtol=1e-8, atol=0, err_msg=f"{name} {k} {f}")
            assert x["supervoxelNum"] == y["supervoxelNum"]
    assert swapped < 20
