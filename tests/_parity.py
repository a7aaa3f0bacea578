"""The parity check every GPU test applies: the CUDA path's outputs against the FP64
oracle's on the same inputs.

kNN candidate lists and supervoxel assignments exact; responsibilities 1e-5 absolute;
means 1e-3 voxel; precision matrices 1e-4 relative (to the largest entry of each matrix);
beta, nu, alpha 1e-9; log-likelihood 1e-6 relative with the mixed-precision voxel terms
(1e-9 with FP64 voxel terms, passed by the caller).
"""
import numpy as np

RNK_TOL = 1e-5
M_TOL = 1e-3
W_RTOL = 1e-4


def errors(g, o):
    """The largest errors of a run g against the oracle's run o (live Gaussians only)."""
    gg, og = g["gauss"], o["gauss"]
    a = og["m_o"][:, 0] > -1e31
    wscale = np.max(np.abs(og["W_k"][a]), axis=1, keepdims=True)
    return dict(ind_equal=bool(np.array_equal(g["ind"], o["ind"])),
                rnk=float(np.max(np.abs(g["rnk"] - o["rnk"]))),
                m=float(np.max(np.abs(gg["m_k"][a] - og["m_k"][a]))) if a.any() else 0.0,
                w_rel=float(np.max(np.abs(gg["W_k"][a] - og["W_k"][a]) / wscale)) if a.any() else 0.0,
                ll_rel=abs(g["ll"] - o["ll"]) / abs(o["ll"]))


def compare(g, o, ll_rtol=1e-6):
    assert g["iterations"] == o["iterations"]
    np.testing.assert_array_equal(g["ind"], o["ind"])
    assert np.max(np.abs(g["rnk"] - o["rnk"])) <= RNK_TOL
    gg, og = g["gauss"], o["gauss"]
    alive_g = gg["m_o"][:, 0] > -1e31
    alive_o = og["m_o"][:, 0] > -1e31
    np.testing.assert_array_equal(alive_g, alive_o)
    np.testing.assert_array_equal(gg["supervoxelNum"], og["supervoxelNum"])
    for k in range(gg.shape[0]):
        n = og["supervoxelNum"][k]
        np.testing.assert_array_equal(gg["supervoxelIdx"][k][:n], og["supervoxelIdx"][k][:n])
    a = alive_o
    assert np.max(np.abs(gg["m_k"][a] - og["m_k"][a])) <= M_TOL
    wscale = np.max(np.abs(og["W_k"][a]), axis=1, keepdims=True)
    assert np.max(np.abs(gg["W_k"][a] - og["W_k"][a]) / wscale) <= W_RTOL
    for key in ("nu_k", "beta_k", "alpha_k"):
        np.testing.assert_allclose(gg[key][a], og[key][a], rtol=1e-9, atol=1e-9)
    assert abs(g["ll"] - o["ll"]) <= ll_rtol * abs(o["ll"])
    assert abs(g["ll_true"] - o["ll_true"]) <= ll_rtol * abs(o["ll_true"])
    assert abs(g["ll_as_reference"] - o["ll_as_reference"]) <= ll_rtol * abs(o["ll_as_reference"])
    assert g["n_dead"] == o["n_dead"]
