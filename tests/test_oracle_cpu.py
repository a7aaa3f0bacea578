"""CPU checks of the oracle's building blocks against independent numpy/scipy
computations, and of the algebra the CUDA path relies on (the moment form of the E-step and
M-step), so that the checker itself is checked."""
import ctypes as C

import numpy as np
import pytest

import _fixtures as F
from oracle import oracle as O

VP = C.c_void_p


def lib():
    lb = O.lib()
    lb.or_det3.argtypes = [VP]
    lb.or_det3.restype = C.c_double
    lb.or_inv3.argtypes = [VP, VP]
    lb.or_estep.argtypes = [VP, VP, C.c_int64, VP, C.c_int32, VP, C.c_int32, VP, VP]
    lb.or_mstep.argtypes = [VP, VP, C.c_int64, VP, C.c_int32, C.c_int32, VP, VP, C.c_int32, VP, VP, VP]
    lb.or_prior_constants.argtypes = [VP, C.c_int32, C.c_double]
    lb.or_total_alpha.argtypes = [VP, C.c_int32, C.c_int32]
    lb.or_total_alpha.restype = C.c_double
    return lb


def sym(w):
    return np.array([[w[0], w[1], w[2]], [w[1], w[3], w[4]], [w[2], w[4], w[5]]])


def test_digamma_matches_scipy():
    sp = pytest.importorskip("scipy.special")
    xs = np.concatenate([np.geomspace(1e-7, 1e6, 400), -np.linspace(0.01, 20.99, 200) + 1e-3 * np.arange(200) / 200])
    for x in xs:
        assert O.lib().or_digamma(float(x)) == pytest.approx(float(sp.digamma(x)), rel=1e-11, abs=1e-11)
    assert O.lib().or_digamma(-3.0) == -1e300  # pole


def test_det_inverse_and_eig():
    lb = lib()
    rng = np.random.default_rng(0)
    for _ in range(200):
        A = rng.normal(size=(3, 3))
        M = A @ A.T + 0.1 * np.eye(3)
        w = np.array([M[0, 0], M[0, 1], M[0, 2], M[1, 1], M[1, 2], M[2, 2]])
        assert lb.or_det3(w.ctypes.data) == pytest.approx(np.linalg.det(M), rel=1e-10)
        inv = np.zeros(6)
        lb.or_inv3(w.ctypes.data, inv.ctypes.data)
        np.testing.assert_allclose(sym(inv), np.linalg.inv(M), rtol=1e-9, atol=1e-12)
        d = np.zeros(3)
        v = np.zeros(9)
        lb.or_eig3(w.ctypes.data, d.ctypes.data, v.ctypes.data)
        np.testing.assert_allclose(np.sort(d), np.linalg.eigvalsh(M), rtol=1e-9, atol=1e-12)
        V = v.reshape(3, 3)  # rows are eigenvectors
        np.testing.assert_allclose(V.T @ np.diag(d) @ V, M, rtol=1e-8, atol=1e-10)
        assert d[0] >= d[2] >= d[1] - 1e-12  # largest, smallest, middle


def test_eig_of_isotropic_matrix_is_nan_like_the_reference():
    # the trigonometric branch divides q by p^1.5 with p = 0 (GMEMupdateCUDA.cu:239): NaN
    # eigenvalues, so the regularised W is NaN and the kill rule removes the Gaussian
    lb = lib()
    w = np.array([2, 0, 0, 2, 0, 2], float)
    d = np.zeros(3)
    v = np.zeros(9)
    lb.or_eig3(w.ctypes.data, d.ctypes.data, v.ctypes.data)
    assert np.isnan(d).all()


def test_eig_degenerate_cases_reconstruct():
    lb = lib()
    for w in ([3, 0, 0, 1, 0, 1], [1, 0.5, 0, 1, 0, 0.3], [0, 0, 0, 0, 0, 0], [1, 0, 0, 1, 0, 0]):
        w = np.array(w, float)
        d = np.zeros(3)
        v = np.zeros(9)
        lb.or_eig3(w.ctypes.data, d.ctypes.data, v.ctypes.data)
        V = v.reshape(3, 3)
        np.testing.assert_allclose(V.T @ np.diag(d) @ V, sym(w), atol=1e-9)


def test_knn_canonical_matches_brute_force():
    rng = np.random.default_rng(1)
    nq, nr = 400, 150
    q = rng.uniform(0, 50, size=(3, nq)).astype(np.float32)
    r = rng.uniform(0, 50, size=(nr, 3)).astype(np.float32)
    r[3] = r[7]  # an exact tie
    s = np.array([1, 1, 2], np.float32)
    got = O.knn(q.reshape(-1), r.reshape(-1)).reshape(5, nq)
    for i in range(nq):
        a = (q[:, i][None, :] - r) * s
        d = (a[:, 0] * a[:, 0]).astype(np.float32)
        d = np.float32(a[:, 1]) * a[:, 1] + d  # fma differences are below the ordering here
        d = np.float32(a[:, 2]) * a[:, 2] + d
        order = np.lexsort((np.arange(nr), d))[:5]
        assert set(order) == set(got[:, i]) or np.allclose(np.sort(d[order]), np.sort(d[got[:, i]]))
        assert all(got[j, i] < got[j + 1, i] or d[got[j, i]] < d[got[j + 1, i]] for j in range(4))


def test_knn_reference_rule_same_sets_when_distances_differ():
    rng = np.random.default_rng(2)
    q = rng.uniform(0, 80, size=3 * 300).astype(np.float32)
    r = rng.uniform(0, 80, size=3 * 200).astype(np.float32)
    a = np.sort(O.knn(q, r).reshape(5, -1), axis=0)
    b = np.sort(O.knn(q, r, reference_rule=True).reshape(5, -1), axis=0)
    np.testing.assert_array_equal(a, b)


def _estep_L(frame):
    lb = lib()
    g = np.ascontiguousarray(frame.gauss).copy()
    S, N, K = frame.n_sv, frame.n_vox, g.shape[0]
    ref = np.ascontiguousarray(g["m_k"].astype(np.float32)).reshape(-1)
    ind = O.knn(frame.centroids, ref)
    total = lb.or_total_alpha(g.ctypes.data, K, 0)
    lb.or_prior_constants(g.ctypes.data, K, total)
    rnk = np.zeros(5 * S, np.float32)
    L = np.zeros(5 * S)
    lb.or_estep(g.ctypes.data, frame.query.ctypes.data, N, frame.label_ptr.ctypes.data, S, ind.ctypes.data, 0,
                rnk.ctypes.data, L.ctypes.data)
    return g, ind, rnk, L


@pytest.mark.parametrize("name", ["tiny", "small", "hard"])
def test_estep_moment_form_is_the_per_voxel_sum(name):
    """sum_v -1/2(3/beta + nu d'Wd) = -1/2(3n/beta + nu tr(W D)), D from centred moments --
    the identity the CUDA E-step uses -- checked against the oracle's per-voxel FP64 sum."""
    f = F.frame(name)
    g, ind, rnk, L = _estep_L(f)
    S, N = f.n_sv, f.n_vox
    x = f.query.reshape(3, N).astype(np.float64)
    c = f.centroids.reshape(3, S).astype(np.float64)
    for s in range(S):
        a, b = f.label_ptr[s], f.label_ptr[s + 1]
        e = x[:, a:b] - c[:, s:s + 1]
        n = b - a
        G1 = e.sum(axis=1)
        G2 = e @ e.T
        for j in range(5):
            G = g[ind[j * S + s]]
            if G["m_o"][0] < -1e31 or n == 0:
                continue
            u = G["m_k"] - c[:, s]
            D = G2 - np.outer(G1, u) - np.outer(u, G1) + n * np.outer(u, u)
            Lm = -0.5 * (3 * n / G["beta_k"] + G["nu_k"] * np.sum(sym(G["W_k"]) * D)) + n * (G["eLR"] + 0.5 * G["eLD"])
            assert Lm == pytest.approx(L[j * S + s], rel=1e-10, abs=1e-8)


@pytest.mark.parametrize("name", ["small", "hard"])
def test_mstep_moment_form_is_the_weighted_sum(name):
    f = F.frame(name)
    g, ind, rnk, L = _estep_L(f)
    lb = lib()
    S, N, K = f.n_sv, f.n_vox, g.shape[0]
    Nk, Xk, Sk = np.zeros(K), np.zeros(3 * K), np.zeros(6 * K)
    lb.or_mstep(f.query.ctypes.data, f.img.ctypes.data, N, f.label_ptr.ctypes.data, S, K, ind.ctypes.data,
                rnk.ctypes.data, 0, Nk.ctypes.data, Xk.ctypes.data, Sk.ctypes.data)
    x = f.query.reshape(3, N).astype(np.float64)
    c = f.centroids.reshape(3, S).astype(np.float64)
    I = f.img.astype(np.float64)
    A0, A1, A2 = np.zeros(K), np.zeros((K, 3)), np.zeros((K, 3, 3))
    for s in range(S):
        a, b = f.label_ptr[s], f.label_ptr[s + 1]
        e = x[:, a:b] - c[:, s:s + 1]
        H0 = I[a:b].sum()
        H1 = (I[a:b] * e).sum(axis=1)
        H2 = (I[a:b] * e) @ e.T
        for j in range(5):
            r = float(rnk[j * S + s])
            if not r > 1e-3:
                continue
            k = ind[j * S + s]
            d = c[:, s]  # re-centre at the origin
            A0[k] += r * H0
            A1[k] += r * (H1 + H0 * d)
            A2[k] += r * (H2 + np.outer(H1, d) + np.outer(d, H1) + H0 * np.outer(d, d))
    ok = A0 > 0
    np.testing.assert_allclose(A0, Nk, rtol=1e-11, atol=1e-12)
    mean = A1[ok] / A0[ok, None]
    np.testing.assert_allclose(mean, Xk.reshape(K, 3)[ok], rtol=1e-9, atol=1e-9)
    scat = A2[ok] - np.einsum("ki,kj->kij", A1[ok], A1[ok]) / A0[ok, None, None]
    want = Sk.reshape(K, 6)[ok]
    got = np.stack([scat[:, 0, 0], scat[:, 0, 1], scat[:, 0, 2], scat[:, 1, 1], scat[:, 1, 2], scat[:, 2, 2]], 1)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max())


@pytest.mark.parametrize("name", ["tiny", "small", "hard", "big"])
def test_fp64_and_ref32_modes_agree_to_float_precision(name):
    f = F.frame(name)
    a = O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, O.params(max_iter=5, tol=-1))
    b = O.em_run(f.query, f.img, f.centroids, f.label_ptr, f.gauss, O.params(max_iter=5, tol=-1, mode=O.MODE_REF32))
    np.testing.assert_array_equal(np.sort(a["ind"].reshape(5, -1), 0), np.sort(b["ind"].reshape(5, -1), 0))
    alive = a["gauss"]["m_o"][:, 0] > -1e31
    np.testing.assert_array_equal(alive, b["gauss"]["m_o"][:, 0] > -1e31)
    assert np.max(np.abs(a["gauss"]["m_k"][alive] - b["gauss"]["m_k"][alive])) < 5e-3
    assert a["ll_as_reference"] == pytest.approx(b["ll_as_reference"], rel=1e-4)


def test_update_priors_matches_reference_formula():
    g = F.frame("small").gauss.copy()
    g["nu_o"] = g["nu_k"] * 0.25
    ref = g.copy()
    O.lib().or_update_priors(g.ctypes.data, g.shape[0], 0.01, 1.0, 0.8, 1234.5)
    n = ref["nu_k"] - ref["nu_o"]
    np.testing.assert_allclose(g["beta_o"], np.maximum(0.01 * n, 1e-5))
    np.testing.assert_allclose(g["nu_o"], np.maximum(n, 3.0))
    np.testing.assert_allclose(g["alpha_o"], 1234.5 * 1e-5 * 0.8)
    np.testing.assert_allclose(g["W_o"], ref["W_k"] * (ref["nu_k"] / g["nu_o"])[:, None])
    np.testing.assert_allclose(g["nu_k"], 2 * ref["nu_k"])
    np.testing.assert_allclose(g["W_k"], ref["W_k"] / 2)
    np.testing.assert_array_equal(g["m_o"], ref["m_k"])


def test_supervoxel_knn_topk_restatement():
    """The tracking graph's supervoxel kNN restated in the oracle (k <= 11, distances): its
    first five are the canonical 5-NN, shorter lists are prefixes of longer ones, and slots
    beyond the reference points are -1 / 1e32."""
    rng = np.random.default_rng(3)
    q = rng.uniform(0, 100, size=(3, 300)).astype(np.float32).reshape(-1)
    r = rng.uniform(0, 100, size=(3, 200)).astype(np.float32)
    ind11, d11 = O.knn_topk(q, r.reshape(-1), 11)
    ind5, d5 = O.knn_topk(q, r.reshape(-1), 5)
    np.testing.assert_array_equal(ind5, O.knn(q, np.ascontiguousarray(r.T).reshape(-1)))
    np.testing.assert_array_equal(ind11.reshape(11, -1)[:5], ind5.reshape(5, -1))
    np.testing.assert_array_equal(d11.reshape(11, -1)[:5], d5.reshape(5, -1))
    assert np.all(np.diff(d11.reshape(11, -1), axis=0) >= 0)
    ind, d = O.knn_topk(q, r[:, :3].reshape(-1), 5)
    assert np.all(ind.reshape(5, -1)[3:] == -1) and np.all(d.reshape(5, -1)[3:] == np.float32(1e32))
