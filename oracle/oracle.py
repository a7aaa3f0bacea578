"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU oracle (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")

MODE_FP64 = 0
MODE_REF32 = 1
LL_AS_REFERENCE = 0
LL_TRUE = 1


class OrParams(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("w4dof", C.c_int32), ("tol", C.c_double), ("lambda_min", C.c_double),
                ("lambda_max", C.c_double), ("max_exc", C.c_double), ("scale", C.c_float * 3),
                ("ll_mode", C.c_int32), ("mode", C.c_int32)]


class OrStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("ll", C.c_double), ("ll_true", C.c_double),
                ("ll_as_reference", C.c_double), ("total_alpha", C.c_double), ("n_dead", C.c_int32)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            build()
        _lib = C.CDLL(SO)
        vp = C.c_void_p
        _lib.or_em_run.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_int32, vp, C.c_int32, C.POINTER(OrParams), vp,
                                   vp, vp, C.POINTER(OrStats)]
        _lib.or_em_run.restype = C.c_int
        _lib.or_knn_canonical.argtypes = [vp, C.c_int64, vp, C.c_int32, C.POINTER(C.c_float), vp]
        _lib.or_knn_topk.argtypes = [vp, C.c_int64, vp, C.c_int32, C.c_int32, C.POINTER(C.c_float), vp, vp]
        _lib.or_knn_reference.argtypes = [vp, C.c_int64, vp, C.c_int32, C.POINTER(C.c_float), vp]
        _lib.or_digamma.argtypes = [C.c_double]
        _lib.or_digamma.restype = C.c_double
        _lib.or_eig3.argtypes = [vp, vp, vp]
        _lib.or_regularize.argtypes = [vp, C.c_int32, C.POINTER(C.c_float), C.c_int32, C.c_double, C.c_double,
                                       C.c_double]
        _lib.or_update_priors.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]
        _lib.or_local_likelihood.argtypes = [vp, C.c_int32, vp, vp, C.c_int64, vp, C.c_int32, vp, vp, vp, C.c_int32,
                                             C.c_int32, vp]
        _lib.or_local_likelihood.restype = C.c_int
        _lib.or_split_proposal.argtypes = [vp, C.POINTER(C.c_float), vp, vp]
        _lib.or_set_num_threads.argtypes = [C.c_int]
        _lib.or_num_threads.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data


def params(max_iter=20, tol=0.0, scale=(1.0, 1.0, 2.0), w4dof=1, ll_mode=LL_AS_REFERENCE, mode=MODE_FP64,
           lambda_min=0.02, lambda_max=0.2222, max_exc=9.0):
    p = OrParams()
    p.max_iter, p.w4dof, p.tol = max_iter, w4dof, tol
    p.lambda_min, p.lambda_max, p.max_exc = lambda_min, lambda_max, max_exc
    p.scale[:] = list(scale)
    p.ll_mode, p.mode = ll_mode, mode
    return p


def em_run(query, img, cent, lptr, gauss, p: OrParams, threads: int = 0):
    """Run the oracle EM; gauss (structured 288-byte records) is copied, not modified."""
    lb = lib()
    if threads:
        lb.or_set_num_threads(threads)
    g = np.ascontiguousarray(gauss).copy()
    if g.dtype.itemsize != 288:
        raise ValueError("Gaussian records must be the 288-byte GaussianMixtureModelCUDA layout")
    S = lptr.shape[0] - 1
    N = img.shape[0]
    rnk = np.zeros(5 * S, np.float32)
    ind = np.zeros(5 * S, np.int32)
    hist = np.zeros(max(p.max_iter, 1), np.float64)
    st = OrStats()
    rc = lb.or_em_run(_p(query), _p(img), _p(cent), _p(lptr), N, S, _p(g), g.shape[0], C.byref(p), _p(rnk), _p(ind),
                      _p(hist), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle em_run failed ({rc})")
    return dict(gauss=g, rnk=rnk, ind=ind, ll_hist=hist[:st.iterations], iterations=st.iterations,
                converged=st.converged, ll=st.ll, ll_true=st.ll_true, ll_as_reference=st.ll_as_reference,
                total_alpha=st.total_alpha, n_dead=st.n_dead)


def split_proposal(rec, scale=(1.0, 1.0, 2.0)):
    """The principal-axis split of one 288-byte record (GaussianMixtureModel::splitGaussian
    and updatePriorsAfterSplitProposal on both halves): (the split Gaussian, the new one)."""
    g = np.ascontiguousarray(np.asarray(rec).reshape(1)).copy()
    a, b = g.copy(), g.copy()
    sc = (C.c_float * 3)(*scale)
    lib().or_split_proposal(_p(g), sc, _p(a), _p(b))
    return a[0], b[0]


def split_round(query, img, cent, lptr, gauss, ind, cand, p: OrParams):
    """The split round restated (mainTrackingGaussianMixtureModel.cpp:1233-1507, candidates
    given): the local log-likelihood of each candidate's supervoxels before, the principal-axis
    split of each candidate (the new Gaussian appended), every other Gaussian fixed, the EM on
    the split mixture, the local log-likelihood of the same supervoxels after."""
    g = np.ascontiguousarray(gauss).copy()
    K = g.shape[0]
    lists = [[int(s) for s in g["supervoxelIdx"][k][:g["supervoxelNum"][k]]] for k in cand]
    before = local_likelihood(query, img, lptr, ind, g, lists)
    g2 = np.zeros(K + len(cand), g.dtype)  # (np.concatenate would drop the record's padding)
    g2[:K] = g
    for k in range(K):
        if k not in set(cand):
            g2["fixed"][k] = 1
    scale = tuple(p.scale)
    for i, k in enumerate(cand):
        a, b = split_proposal(g2[k], scale)
        g2[k] = a
        g2[K + i] = b
    out = em_run(query, img, cent, lptr, g2, p)
    after = local_likelihood(query, img, lptr, out["ind"], out["gauss"], lists)
    return dict(before=before, after=after, split=g2, **out)


REF_GMM_SO = os.path.join(HERE, "_ref", "libtgmm_ref_gmm.so")
_ref_gmm = None


def ref_gmm_available() -> bool:
    return os.path.exists(REF_GMM_SO)


def ref_split_gaussian(rec, scale=(1.0, 1.0, 2.0)):
    """The reference's own GaussianMixtureModel::splitGaussian(GM, id) and
    updatePriorsAfterSplitProposal (host code, compiled from its sources)."""
    global _ref_gmm
    if _ref_gmm is None:
        _ref_gmm = C.CDLL(REF_GMM_SO)
        _ref_gmm.ref_split_gaussian.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
        _ref_gmm.ref_split_gaussian.restype = C.c_int
    g = np.ascontiguousarray(np.asarray(rec).reshape(1)).copy()
    a, b = g.copy(), g.copy()
    sc = (C.c_float * 3)(*scale)
    if _ref_gmm.ref_split_gaussian(_p(g), sc, _p(a), _p(b)) != 0:
        raise RuntimeError("reference split failed")
    return a[0], b[0]


def lists_csr(lists):
    """A list of supervoxel-index lists as CSR arrays (list_ptr int32, list_idx int32)."""
    ptr = np.zeros(len(lists) + 1, np.int32)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    idx = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in lists]) if ptr[-1] else
                               np.zeros(1, np.int32))
    return ptr, idx


def local_likelihood(query, img, lptr, ind, gauss, lists, mode=MODE_FP64):
    """The local log-likelihood of each supervoxel list (calculateLocalLikelihood) under the
    Gaussians `gauss` with each supervoxel's candidates `ind` (slot-major, 5*S)."""
    g = np.ascontiguousarray(gauss)
    lp = np.ascontiguousarray(lptr, np.int64)
    ind = np.ascontiguousarray(ind, np.int32)
    ptr, idx = lists_csr(lists)
    out = np.zeros(len(lists), np.float64)
    rc = lib().or_local_likelihood(_p(g), g.shape[0], _p(np.ascontiguousarray(query, np.float32)),
                                   _p(np.ascontiguousarray(img, np.float32)), img.shape[0], _p(lp), lp.shape[0] - 1,
                                   _p(ind), _p(ptr), _p(idx), len(lists), mode, _p(out))
    if rc != 0:
        raise ValueError("local_likelihood: supervoxel or candidate index out of range")
    return out


def knn(query, ref_xyz, scale=(1.0, 1.0, 2.0), reference_rule=False):
    lb = lib()
    nq = query.shape[0] // 3
    ind = np.zeros(5 * nq, np.int32)
    sc = (C.c_float * 3)(*scale)
    f = lb.or_knn_reference if reference_rule else lb.or_knn_canonical
    f(_p(query), nq, _p(ref_xyz), ref_xyz.shape[0] // 3, sc, _p(ind))
    return ind


def knn_topk(query, ref_soa, k, scale=(1.0, 1.0, 2.0)):
    """The supervoxel kNN of the tracking graph (k <= 11, distances), canonical order."""
    lb = lib()
    q = np.ascontiguousarray(query, np.float32)
    r = np.ascontiguousarray(ref_soa, np.float32)
    nq, nref = q.shape[0] // 3, r.shape[0] // 3
    ind = np.zeros(k * nq, np.int32)
    dist = np.zeros(k * nq, np.float32)
    sc = (C.c_float * 3)(*scale)
    lb.or_knn_topk(_p(q), nq, _p(r), nref, k, sc, _p(ind), _p(dist))
    return ind, dist


# ---------------------------------------------------------------------------
# The reference's own GPU path, compiled from its sources by oracle/build_ref.sh.
# ---------------------------------------------------------------------------
REF_SO = os.path.join(HERE, "_ref", "libtgmm_ref.so")
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        vp = C.c_void_p
        _ref.ref_em_run.argtypes = [vp, vp, vp, vp, C.c_longlong, C.c_int, vp, C.c_int, C.c_int, C.c_double, C.c_int,
                                    C.c_double, C.c_double, C.c_double, vp, vp, vp]
        _ref.ref_em_run.restype = C.c_int
        _ref.ref_knn.argtypes = [vp, C.c_longlong, vp, C.c_int, vp, vp]
        _ref.ref_knn.restype = C.c_int
        _ref.ref_write_gmm_xml.argtypes = [C.c_char_p, vp, C.c_int]
        _ref.ref_write_gmm_xml.restype = C.c_int
        _ref.ref_local_likelihood.argtypes = [vp, vp, vp, C.c_longlong, C.c_int, vp, vp, C.c_int, vp, vp, C.c_int, vp]
        _ref.ref_local_likelihood.restype = C.c_int
    return _ref


def ref_em_run(query, img, cent, lptr, gauss, max_iter=20, tol=-1.0, w4dof=1, scale=(1.0, 1.0, 2.0),
               lambda_min=0.02, lambda_max=0.2222, max_exc=9.0):
    """Run the unmodified reference GMEMvariationalInferenceCUDAWithSupervoxels."""
    g = np.ascontiguousarray(gauss).copy()
    if g.dtype.itemsize != 288:
        raise ValueError("Gaussian records must be the 288-byte GaussianMixtureModelCUDA layout")
    q = np.ascontiguousarray(query, np.float32).copy()
    im = np.ascontiguousarray(img, np.float32).copy()
    ce = np.ascontiguousarray(cent, np.float32).copy()
    lp = np.ascontiguousarray(lptr, np.int64).copy()
    S = lp.shape[0] - 1
    sc = np.asarray(scale, np.float32)
    rnk = np.zeros(5 * S, np.float32)
    ind = np.zeros(5 * S, np.int32)
    rc = ref_lib().ref_em_run(_p(q), _p(im), _p(ce), _p(lp), im.shape[0], S, _p(g), g.shape[0], max_iter, tol, w4dof,
                              lambda_min, lambda_max, max_exc, _p(sc), _p(rnk), _p(ind))
    if rc != 0:
        raise RuntimeError(f"reference run failed ({rc})")
    return dict(gauss=g, rnk=rnk, ind=ind)


def pad_supervoxels(cent, lptr, block=1024, far=-1000.0):
    """The frame's supervoxel arrays padded to a multiple of `block` supervoxels with empty
    ones (no voxels; centroid at (far, far, far)).  The reference's kNN kernel, launched with
    blocks of min(1024, S) threads, returns early for the surplus threads of its last block
    and then calls __syncthreads() (knnCuda.cu:69,106 and :154); with S a multiple of 1024
    no thread returns early.  An empty supervoxel adds nothing to the M-step sums, the
    log-likelihood or the assignment (its responsibilities are 1/5 each), so the outputs of the
    real supervoxels do not change (tests/test_gpu_reference.py checks this)."""
    S = lptr.shape[0] - 1
    Sp = -(-S // block) * block
    c = np.full((3, Sp), far, np.float32)
    c[:, :S] = np.asarray(cent, np.float32).reshape(3, S)
    lp = np.full(Sp + 1, lptr[-1], np.int64)
    lp[:S + 1] = lptr
    return c.reshape(-1), lp


def ref_knn(query, ref_xyz, scale=(1.0, 1.0, 2.0)):
    q = np.ascontiguousarray(query, np.float32)
    r = np.ascontiguousarray(ref_xyz, np.float32)
    nq = q.shape[0] // 3
    ind = np.zeros(5 * nq, np.int32)
    sc = np.asarray(scale, np.float32)
    rc = ref_lib().ref_knn(_p(q), nq, _p(r), r.shape[0] // 3, _p(sc), _p(ind))
    if rc != 0:
        raise RuntimeError(f"reference kNN failed ({rc})")
    return ind


def ref_local_likelihood(query, img, lptr, ind, gauss, lists):
    """The reference's own calculateLocalLikelihood (its GPU kernels) on host arrays."""
    g = np.ascontiguousarray(gauss).copy()
    q = np.ascontiguousarray(query, np.float32).copy()
    im = np.ascontiguousarray(img, np.float32).copy()
    lp = np.ascontiguousarray(lptr, np.int64).copy()
    ind = np.ascontiguousarray(ind, np.int32).copy()
    ptr, idx = lists_csr(lists)
    out = np.zeros(len(lists), np.float64)
    rc = ref_lib().ref_local_likelihood(_p(q), _p(im), _p(lp), im.shape[0], lp.shape[0] - 1, _p(ind), _p(g),
                                        g.shape[0], _p(ptr), _p(idx), len(lists), _p(out))
    if rc != 0:
        raise RuntimeError(f"reference local likelihood failed ({rc})")
    return out


def ref_write_gmm_xml(path, gauss):
    """The reference's own GMM XML writer on host records (gauss: 288-byte structured array)."""
    g = np.ascontiguousarray(gauss).copy()
    rc = ref_lib().ref_write_gmm_xml(str(path).encode(), _p(g), g.shape[0])
    if rc != 0:
        raise RuntimeError(f"reference XML writer failed ({rc})")


REF_F3_SO = os.path.join(HERE, "_ref", "libtgmm_ref_f3.so")
_ref_f3 = None


def ref_f3_available() -> bool:
    return os.path.exists(REF_F3_SO)


def ref_knn_k(query, ref_soa, k, scale=(1.0, 1.0, 2.0)):
    """The reference's own supervoxel kNN of the tracking graph (its slot order: replace the
    current maximum, later index on ties); n_query <= 1024."""
    global _ref_f3
    if _ref_f3 is None:
        _ref_f3 = C.CDLL(REF_F3_SO)
        vp = C.c_void_p
        _ref_f3.ref_knn_k.argtypes = [vp, vp, vp, vp, C.c_longlong, C.c_int, C.c_int, vp]
        _ref_f3.ref_knn_k.restype = C.c_int
    q = np.ascontiguousarray(query, np.float32).copy()
    r = np.ascontiguousarray(ref_soa, np.float32).copy()
    nq, nref = q.shape[0] // 3, r.shape[0] // 3
    ind = np.zeros(k * nq, np.int32)
    dist = np.zeros(k * nq, np.float32)
    sc = np.asarray(scale, np.float32)
    rc = _ref_f3.ref_knn_k(_p(ind), _p(dist), _p(q), _p(r), nq, nref, k, _p(sc))
    if rc != 0:
        raise RuntimeError(f"reference supervoxel kNN failed ({rc})")
    return ind, dist


# ---------------------------------------------------------------------------
# Frame preparation from a supervoxel label volume (frame_oracle.c).
# ---------------------------------------------------------------------------
class OrFrameParams(C.Structure):
    _fields_ = [("max_size", C.c_int32), ("max_pct", C.c_float), ("conn", C.c_int32), ("min_size", C.c_int32)]


def frame_params(max_size=3000, max_pct=0.4, conn=6, min_size=50) -> OrFrameParams:
    return OrFrameParams(max_size, max_pct, conn, min_size)


def frame_build(raw, label, n_labels, p: OrFrameParams | None = None, max_vox=None):
    """The EM's input arrays from a raw 16-bit volume and a supervoxel label volume (shape
    (Z, Y, X), labels 1..n_labels, 0 = none).  Returns (rc, dict)."""
    p = p or frame_params()
    raw = np.ascontiguousarray(raw, np.uint16)
    label = np.ascontiguousarray(label, np.uint32)
    Z, Y, X = raw.shape
    dims = np.array([X, Y, Z], np.int32)
    nvol = raw.size if max_vox is None else int(max_vox)
    query = np.zeros(3 * nvol, np.float32)
    img = np.zeros(nvol, np.float32)
    cent = np.zeros(3 * n_labels, np.float32)
    lptr = np.zeros(n_labels + 1, np.int64)
    thr = np.zeros(n_labels, np.uint16)
    n_vox = C.c_int64(0)
    n_sv = C.c_int32(0)
    L = lib()
    vp = C.c_void_p
    L.or_frame_build.argtypes = [vp, vp, vp, C.c_int32, C.POINTER(OrFrameParams), vp, vp, vp, vp, vp, C.c_int64,
                                 C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    L.or_frame_build.restype = C.c_int
    rc = L.or_frame_build(_p(raw), _p(label), _p(dims), n_labels, C.byref(p), _p(query), _p(img), _p(cent), _p(lptr),
                          _p(thr), nvol, n_labels, C.byref(n_vox), C.byref(n_sv))
    N, S = n_vox.value, n_sv.value
    out = dict(n_vox=N, n_sv=S)
    if rc == 0:
        out.update(query=query[:3 * N].copy(), img=img[:N].copy(), cent=cent[:3 * S].copy(),
                   lptr=lptr[:S + 1].copy(), thr=thr[:S].copy())
    return rc, out


def erase_order(erased):
    e = np.ascontiguousarray(erased, np.uint8)
    order = np.zeros(e.shape[0], np.int32)
    L = lib()
    L.or_erase_order.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.or_erase_order(_p(e), e.shape[0], _p(order))
    return order[:e.shape[0] - int((e != 0).sum())]


def supervoxel_lists(label, n_labels):
    """Per label, its voxels' linear indices in ascending order (CSR)."""
    flat = np.ascontiguousarray(label, np.uint32).reshape(-1)
    idx = np.nonzero(flat)[0]
    lab = flat[idx].astype(np.int64) - 1
    order = np.argsort(lab, kind="stable")
    lin = idx[order].astype(np.uint64)
    ptr = np.zeros(n_labels + 1, np.int64)
    np.add.at(ptr, lab + 1, 1)
    return np.cumsum(ptr), lin


REF_F1_SO = os.path.join(HERE, "_ref", "libtgmm_ref_f1.so")


def ref_f1_available() -> bool:
    return os.path.exists(REF_F1_SO)


def ref_trim_stats(raw, ptr, lin, max_size=3000, max_pct=0.4, conn=6):
    """The reference's own trimSupervoxel<uint16>() and weightedGaussianStatistics<uint16>(true)
    (temporalLogicalRules/supervoxel.cpp) on each supervoxel of the CSR (ptr, lin)."""
    ref = C.CDLL(REF_F1_SO)
    vp = C.c_void_p
    ref.ref_trim_stats.argtypes = [vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_float, C.c_int32, vp, vp, vp, vp, vp]
    ref.ref_trim_stats.restype = C.c_int
    raw = np.ascontiguousarray(raw, np.uint16)
    Z, Y, X = raw.shape
    dims = np.array([X, Y, Z], np.int32)
    n = ptr.shape[0] - 1
    ptr = np.ascontiguousarray(ptr, np.int64)
    lin = np.ascontiguousarray(lin, np.uint64)
    thr = np.zeros(n, np.uint16)
    cnt = np.zeros(n, np.int64)
    lin_out = np.zeros(max(1, lin.shape[0]), np.uint64)
    cent = np.zeros(3 * n, np.float32)
    inten = np.zeros(n, np.float32)
    rc = ref.ref_trim_stats(_p(raw), _p(dims), _p(ptr), _p(lin), n, max_size, max_pct, conn, _p(thr), _p(cnt),
                            _p(lin_out), _p(cent), _p(inten))
    if rc != 0:
        raise RuntimeError(f"reference trimming failed ({rc})")
    kept = [lin_out[ptr[s]:ptr[s] + cnt[s]].copy() for s in range(n)]
    return dict(thr=thr, cnt=cnt, lists=kept, cent=cent.reshape(n, 3), intensity=inten)


def ref_erase_order(erased):
    """The reference's own eraseSupervoxelFromCurrentSegmentation: the original index of each
    supervoxel left, in the order it leaves them."""
    ref = C.CDLL(REF_F1_SO)
    ref.ref_erase_order.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    ref.ref_erase_order.restype = C.c_int
    e = np.ascontiguousarray(erased, np.uint8)
    order = np.zeros(max(1, e.shape[0]), np.int32)
    left = ref.ref_erase_order(_p(e), e.shape[0], _p(order))
    return order[:left].copy()


def ref_frame_build(raw, label, n_labels, p: OrFrameParams | None = None, max_vox=None, lists=None):
    """The reference's host frame build run with its own trimming, statistics and erase
    (oracle/ref_f1_harness.cpp); same outputs as frame_build.  lists: (ptr, lin) from
    supervoxel_lists(label, n_labels), the reference's per-supervoxel pixel lists, if already
    made.  Returns (rc, dict)."""
    p = p or frame_params()
    ref = C.CDLL(REF_F1_SO)
    vp = C.c_void_p
    ref.ref_frame_build.argtypes = [vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_float, C.c_int32, C.c_int32, vp, vp, vp,
                                    vp, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    ref.ref_frame_build.restype = C.c_int
    raw = np.ascontiguousarray(raw, np.uint16)
    Z, Y, X = raw.shape
    dims = np.array([X, Y, Z], np.int32)
    ptr, lin = lists if lists is not None else supervoxel_lists(label, n_labels)
    mv = raw.size if max_vox is None else int(max_vox)
    query = np.zeros(3 * mv, np.float32)
    img = np.zeros(mv, np.float32)
    cent = np.zeros(3 * n_labels, np.float32)
    lptr = np.zeros(n_labels + 1, np.int64)
    n_vox, n_sv = C.c_int64(0), C.c_int32(0)
    rc = ref.ref_frame_build(_p(raw), _p(dims), _p(ptr), _p(lin), n_labels, p.max_size, p.max_pct, p.conn, p.min_size,
                             _p(query), _p(img), _p(cent), _p(lptr), mv, C.byref(n_vox), C.byref(n_sv))
    N, S = n_vox.value, n_sv.value
    out = dict(n_vox=N, n_sv=S)
    if rc == 0:
        out.update(query=query[:3 * N].copy(), img=img[:N].copy(), cent=cent[:3 * S].copy(), lptr=lptr[:S + 1].copy())
    return rc, out
