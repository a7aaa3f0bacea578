"""ctypes bindings of the C ABI (include/tgmm_gmem.h) and of the synthetic-data library.

The CUDA engine lives in ``libtgmm_gmem.so`` next to this file (built in-tree by
``tgmm_b200/csrc/Makefile``).  Loading fails loudly when it is missing: there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GMEM_SO = os.path.join(HERE, "libtgmm_gmem.so")
SYNTH_SO = os.path.join(HERE, "libtgmm_synth.so")

TGMM_J = 5
TGMM_MAX_SV = 16

# status codes (tgmm_gmem.h)
TGMM_OK = 0
TGMM_ERR_INVALID_ARG = 1
TGMM_ERR_BAD_SIZE = 2
TGMM_ERR_BAD_CSR = 3
TGMM_ERR_NAN_INPUT = 4
TGMM_ERR_CUDA = 5
TGMM_ERR_OOM = 6
TGMM_ERR_DEVICE_FLAG = 7
TGMM_ERR_NOT_SET = 8
TGMM_ERR_ADMISSION = 9
TGMM_ERR_NO_SUPERVOXEL = 10
TGMM_FRAME_BUILD_STAGES = 8

TGMM_LL_AS_REFERENCE = 0
TGMM_LL_TRUE = 1
TGMM_LLPREC_MIXED = 0
TGMM_LLPREC_FP64 = 1

# TgmmEmStats.device_flags bits (tgmm_gmem.h)
TGMM_FLAG_BAD_CSR = 1
TGMM_FLAG_NAN_INPUT = 2
TGMM_FLAG_FEW_GAUSS = 4
TGMM_FLAG_BUCKET_OVERFLOW = 8
TGMM_FLAG_ASSIGN_OVERFLOW = 16
TGMM_FLAG_CELL_OVERFLOW = 32
TGMM_FLAG_STAGE_TIMEOUT = 64

TGMM_KERNEL_MOMENTS = 0
TGMM_KERNEL_LL_PASS = 2
TGMM_KERNEL_LL_PASS_KNN = 3


class TgmmGaussian(C.Structure):
    _fields_ = [
        ("beta_k", C.c_double), ("nu_k", C.c_double), ("alpha_k", C.c_double),
        ("m_k", C.c_double * 3), ("W_k", C.c_double * 6),
        ("expectedLogDetCovarianceCUDA", C.c_double), ("expectedLogResponsivityCUDA", C.c_double),
        ("splitScore", C.c_double),
        ("beta_o", C.c_double), ("nu_o", C.c_double), ("alpha_o", C.c_double),
        ("m_o", C.c_double * 3), ("W_o", C.c_double * 6),
        ("fixed", C.c_ubyte),
        ("supervoxelIdx", C.c_int32 * TGMM_MAX_SV), ("supervoxelNum", C.c_int32),
    ]


assert C.sizeof(TgmmGaussian) == 288

# numpy view of the 288-byte record (same offsets)
GAUSS_DTYPE = np.dtype({
    "names": ["beta_k", "nu_k", "alpha_k", "m_k", "W_k", "eLD", "eLR", "splitScore", "beta_o", "nu_o",
              "alpha_o", "m_o", "W_o", "fixed", "supervoxelIdx", "supervoxelNum"],
    "formats": ["<f8", "<f8", "<f8", ("<f8", 3), ("<f8", 6), "<f8", "<f8", "<f8", "<f8", "<f8", "<f8",
                ("<f8", 3), ("<f8", 6), "u1", ("<i4", 16), "<i4"],
    "offsets": [0, 8, 16, 24, 48, 96, 104, 112, 120, 128, 136, 144, 168, 216, 220, 284],
    "itemsize": 288,
})


class TgmmEmParams(C.Structure):
    _fields_ = [
        ("max_iter_em", C.c_int32), ("w4dof", C.c_int32), ("tol_likelihood", C.c_double),
        ("lambda_min", C.c_double), ("lambda_max", C.c_double), ("max_excentricity", C.c_double),
        ("scale", C.c_float * 3), ("reg_scale", C.c_float * 3),
        ("ll_mode", C.c_int32), ("ll_precision", C.c_int32), ("frame", C.c_int32),
    ]


class TgmmFrame(C.Structure):
    _fields_ = [
        ("query", C.c_void_p), ("img", C.c_void_p), ("centroids", C.c_void_p), ("label_ptr", C.c_void_p),
        ("n_vox", C.c_int64), ("n_sv", C.c_int32), ("n_gauss", C.c_int32),
    ]


class TgmmEmStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("converged", C.c_int32), ("ll", C.c_double), ("ll_true", C.c_double),
        ("ll_as_reference", C.c_double), ("total_alpha", C.c_double), ("n_dead", C.c_int32),
        ("device_flags", C.c_int32), ("knn_searches", C.c_int32), ("reserved", C.c_int32),
    ]


class TgmmPlanDesc(C.Structure):
    _fields_ = [
        ("max_vox", C.c_int64), ("max_sv", C.c_int32), ("max_gauss", C.c_int32), ("max_frames", C.c_int32),
        ("device", C.c_int32),
    ]


class TgmmSynthConfig(C.Structure):
    _fields_ = [
        ("dims", C.c_int32 * 3), ("axis_min", C.c_float), ("axis_max", C.c_float), ("anisotropy", C.c_float),
        ("peak_min", C.c_float), ("peak_max", C.c_float), ("background", C.c_float), ("threshold", C.c_float),
        ("jitter", C.c_float), ("min_size", C.c_int32),
    ]


class TgmmFrameBuildParams(C.Structure):
    _fields_ = [("max_nuclei_size", C.c_int32), ("max_percentile", C.c_float), ("conn3d", C.c_int32),
                ("min_nuclei_size", C.c_int32)]


class TgmmServerDesc(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("hbm_budget", C.c_int64), ("lanes", C.c_int32), ("max_batch_frames", C.c_int32),
        ("max_batch_vox", C.c_int64), ("max_batch_sv", C.c_int32), ("max_batch_gauss", C.c_int32),
        ("params", TgmmEmParams), ("beta_pct", C.c_double), ("nu_pct", C.c_double), ("alpha_pct", C.c_double),
    ]


class TgmmServeRequest(C.Structure):
    _fields_ = [
        ("lineage", C.c_int32), ("tag", C.c_uint64), ("query", C.c_void_p), ("img", C.c_void_p),
        ("centroids", C.c_void_p), ("label_ptr", C.c_void_p), ("n_vox", C.c_int64), ("n_sv", C.c_int32),
        ("rnk_out", C.c_void_p), ("ind_out", C.c_void_p), ("gm_out", C.c_void_p), ("lin", C.c_void_p),
        ("raw", C.c_void_p), ("dims", C.c_int32 * 3), ("raw_offset", C.c_double), ("raw_denom", C.c_double),
        ("run_ptr", C.c_void_p), ("run_start", C.c_void_p), ("run_len", C.c_void_p), ("n_runs", C.c_int64),
    ]


class TgmmServeResult(C.Structure):
    _fields_ = [
        ("tag", C.c_uint64), ("lineage", C.c_int32), ("status", C.c_int32), ("stats", TgmmEmStats),
        ("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double), ("batch_id", C.c_int32),
        ("batch_frames", C.c_int32),
    ]


class TgmmServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("completed", C.c_int64), ("rejected", C.c_int64), ("batches", C.c_int64),
        ("frames_in_batches", C.c_int64), ("hbm_budget", C.c_int64), ("hbm_in_use", C.c_int64),
        ("hbm_peak", C.c_int64), ("h2d_bytes", C.c_int64), ("queued", C.c_int32), ("in_flight", C.c_int32),
    ]


# every function declared in include/tgmm_gmem.h and include/tgmm_serve.h: name -> (restype, argtypes)
_VP = C.c_void_p
GMEM_FUNCS = {
    "tgmm_default_params": (None, [C.POINTER(TgmmEmParams)]),
    "tgmm_plan_create": (C.c_int, [C.POINTER(TgmmPlanDesc), C.POINTER(_VP)]),
    "tgmm_plan_destroy": (C.c_int, [_VP]),
    "tgmm_plan_bytes": (C.c_int64, [C.POINTER(TgmmPlanDesc)]),
    "tgmm_em_run": (C.c_int, [_VP, C.POINTER(TgmmFrame), _VP, _VP, _VP, _VP, C.POINTER(TgmmEmParams),
                              C.POINTER(TgmmEmStats), _VP]),
    "tgmm_em_run_device": (C.c_int, [_VP, C.POINTER(TgmmFrame), _VP, _VP, _VP, C.POINTER(TgmmEmParams),
                                     C.POINTER(TgmmEmStats), _VP]),
    "tgmm_em_run_batch": (C.c_int, [_VP, C.c_int32, C.POINTER(TgmmFrame), C.POINTER(_VP), C.POINTER(_VP),
                                    C.POINTER(_VP), C.POINTER(TgmmEmParams), C.POINTER(TgmmEmStats), _VP]),
    "tgmm_knn": (C.c_int, [_VP, C.c_int64, _VP, C.c_int32, C.POINTER(C.c_float), _VP, _VP]),
    "tgmm_knn_noalloc": (C.c_int, [_VP, C.c_int64, _VP, C.c_int32, C.POINTER(C.c_float), _VP, _VP]),
    "tgmm_local_likelihood": (C.c_int, [C.POINTER(TgmmFrame), _VP, _VP, C.c_int32, _VP, _VP, C.c_int32, _VP, _VP]),
    "tgmm_split_proposal": (C.c_int, [_VP, C.POINTER(C.c_float), _VP, _VP]),
    "tgmm_frame_expand": (C.c_int, [_VP, _VP, C.c_int64, C.POINTER(C.c_int32), C.c_double, C.c_double, _VP, _VP,
                                    _VP]),
    "tgmm_frame_expand_runs": (C.c_int, [_VP, _VP, _VP, _VP, _VP, C.c_int32, C.c_int64, C.c_int64,
                                         C.POINTER(C.c_int32), C.c_double, C.c_double, _VP, _VP, _VP]),
    "tgmm_split_round": (C.c_int, [_VP, C.POINTER(TgmmFrame), _VP, C.c_int32, _VP, _VP, C.c_int32, _VP, _VP,
                                   C.POINTER(TgmmEmParams), _VP, _VP, C.POINTER(TgmmEmStats), _VP]),
    "tgmm_update_priors": (C.c_int, [_VP, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                                     _VP]),
    "tgmm_frame_upload": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int64, C.c_int32, C.POINTER(TgmmFrame)]),
    "tgmm_frame_release": (C.c_int, [C.POINTER(TgmmFrame)]),
    "tgmm_assign_supervoxels": (C.c_int, [_VP, _VP, C.c_int32, _VP, C.c_int32]),
    "tgmm_write_rnk_file": (C.c_int, [C.c_char_p, _VP, _VP, C.c_int32]),
    "tgmm_write_gmm_xml": (C.c_int, [C.c_char_p, _VP, C.c_int32]),
    "tgmm_knn_k": (C.c_int, [_VP, C.c_int64, _VP, C.c_int32, C.c_int32, C.POINTER(C.c_float), _VP, _VP, _VP]),
    "tgmm_frame_build_default_params": (None, [C.POINTER(TgmmFrameBuildParams)]),
    "tgmm_frame_build_bytes": (C.c_int64, [_VP, C.c_int32]),
    "tgmm_frame_build_lists_bytes": (C.c_int64, [_VP, C.c_int32, C.c_int64]),
    "tgmm_frame_build_lists": (C.c_int, [_VP, _VP, _VP, C.c_int64, _VP, C.c_int32, C.POINTER(TgmmFrameBuildParams),
                                         _VP, C.c_int64, _VP, _VP, _VP, _VP, _VP, C.c_int64, C.c_int32,
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int32), _VP, _VP]),
    "tgmm_frame_build": (C.c_int, [_VP, _VP, _VP, C.c_int32, C.POINTER(TgmmFrameBuildParams), _VP, C.c_int64, _VP,
                                   _VP, _VP, _VP, _VP, C.c_int64, C.c_int32, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int32), _VP]),
    "tgmm_frame_build_timed": (C.c_int, [_VP, _VP, _VP, C.c_int32, C.POINTER(TgmmFrameBuildParams), _VP, C.c_int64,
                                         _VP, _VP, _VP, _VP, _VP, C.c_int64, C.c_int32, C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int32), _VP, _VP]),
    "tgmm_plan_time_kernel": (C.c_int, [_VP, C.c_int32, C.c_int32, C.POINTER(C.c_float), _VP]),
    "tgmm_plan_set_knn_group": (C.c_int, [_VP, C.c_int32]),
    "tgmm_plan_set_knn_fusion": (C.c_int, [_VP, C.c_int32]),
    "tgmm_plan_set_stage_wait": (C.c_int, [_VP, C.c_int64]),
    "tgmm_plan_tuning": (C.c_int, [_VP, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "tgmm_plan_autotune": (C.c_int, [_VP, C.c_int32, C.POINTER(TgmmFrame), C.POINTER(_VP), C.POINTER(_VP),
                                     C.POINTER(_VP), C.POINTER(TgmmEmParams), C.c_int32, C.POINTER(C.c_int32), _VP]),
    "tgmm_server_default_desc": (None, [C.POINTER(TgmmServerDesc)]),
    "tgmm_server_create": (C.c_int, [C.POINTER(TgmmServerDesc), C.POINTER(_VP)]),
    "tgmm_server_destroy": (C.c_int, [_VP]),
    "tgmm_server_open_lineage": (C.c_int, [_VP, _VP, C.c_int32, C.POINTER(C.c_int32)]),
    "tgmm_server_close_lineage": (C.c_int, [_VP, C.c_int32]),
    "tgmm_server_read_lineage": (C.c_int, [_VP, C.c_int32, _VP]),
    "tgmm_server_submit": (C.c_int, [_VP, C.POINTER(TgmmServeRequest)]),
    "tgmm_server_poll": (C.c_int, [_VP, C.POINTER(TgmmServeResult), C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "tgmm_server_stats": (C.c_int, [_VP, C.POINTER(TgmmServerStats)]),
    "tgmm_server_selftest": (C.c_int, []),
    "tgmm_last_error": (C.c_char_p, []),
    "tgmm_version": (C.c_char_p, []),
}

SYNTH_FUNCS = {
    "tgmm_synth_nuclei": (None, [C.POINTER(TgmmSynthConfig), C.c_int32, C.c_uint64, _VP, _VP, _VP, _VP]),
    "tgmm_synth_frame": (_VP, [C.POINTER(TgmmSynthConfig), C.c_int32, _VP, _VP, _VP, _VP, C.c_uint64]),
    "tgmm_synth_n_vox": (C.c_int64, [_VP]),
    "tgmm_synth_n_sv": (C.c_int32, [_VP]),
    "tgmm_synth_max_fg": (C.c_float, [_VP]),
    "tgmm_synth_copy": (None, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "tgmm_synth_copy_raw": (None, [_VP, _VP]),
    "tgmm_synth_free": (None, [_VP]),
    "tgmm_synth_init_gaussians": (C.c_int32, [_VP, C.POINTER(TgmmSynthConfig), C.c_int32, _VP, C.c_uint64,
                                              C.POINTER(TgmmEmParams), _VP, _VP]),
}

_gmem = None
_synth = None


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def gmem():
    """The CUDA engine library (raises if it was not built)."""
    global _gmem
    if _gmem is None:
        if not os.path.exists(GMEM_SO):
            raise RuntimeError(f"{GMEM_SO} is missing: build it with `make -C tgmm_b200/csrc` "
                               "(there is no CPU fallback for the EM engine)")
        _gmem = _bind(C.CDLL(GMEM_SO), GMEM_FUNCS)
    return _gmem


def synth():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_SO):
            raise RuntimeError(f"{SYNTH_SO} is missing: build it with `make -C tgmm_b200/csrc`")
        _synth = _bind(C.CDLL(SYNTH_SO), SYNTH_FUNCS)
    return _synth


class TgmmError(RuntimeError):
    def __init__(self, code, where):
        msg = gmem().tgmm_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def check(code, where):
    if code != TGMM_OK:
        raise TgmmError(code, where)


def default_params(**overrides) -> TgmmEmParams:
    """The values tgmm_default_params fills in (the reference defaults,
    parseConfigFile.h:152-195), set here without loading the engine library, so that
    code which only generates data or runs the CPU arithmetic never maps it."""
    p = TgmmEmParams()
    p.max_iter_em, p.w4dof, p.tol_likelihood = 400, 1, 1e-6
    p.lambda_min, p.lambda_max, p.max_excentricity = 0.02, 0.2222, 9.0
    p.scale[:] = [1.0, 1.0, 1.0]
    p.reg_scale[:] = [0.0, 0.0, 0.0]
    p.ll_mode, p.ll_precision, p.frame = TGMM_LL_AS_REFERENCE, TGMM_LLPREC_MIXED, 0
    for k, v in overrides.items():
        if k in ("scale", "reg_scale"):
            getattr(p, k)[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


def records(g) -> np.ndarray:
    """A contiguous copy of Gaussian records in the 288-byte layout with every padding byte
    zero (numpy leaves the three bytes after `fixed` uninitialised in a converted copy, which
    would make equal records compare unequal as bytes)."""
    g = np.asarray(g)
    out = np.zeros(g.shape, GAUSS_DTYPE)
    for name in GAUSS_DTYPE.names:
        out[name] = g[name]
    return out


def records_equal(a, b) -> bool:
    """Every named field of two record arrays equal bit for bit (padding bytes ignored)."""
    a, b = np.asarray(a), np.asarray(b)
    for name in GAUSS_DTYPE.names:
        x, y = np.ascontiguousarray(a[name]), np.ascontiguousarray(b[name])
        if x.shape != y.shape or x.tobytes() != y.tobytes():
            return False
    return True


def ptr(a) -> int:
    """Address of a numpy array or a torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
