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
