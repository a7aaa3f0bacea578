"""CPU checks of the C ABI library: it loads without a GPU, exports every entry point the
headers declare (the C ABI and the reference's mangled C++ names), keeps the 288-byte record
layout, and its host-only functions behave like the reference's post-loop code."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from tgmm_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")

# the reference's C++ entry points, as the reference itself mangles them (g++, cxx11 ABI)
LEGACY_SYMBOLS = [
    "_Z13setDeviceCUDAi",
    "_Z14knnCUDAinPlacePiPfS0_xi",
    "_Z8knnCUDA_PiPfS0_S0_xiiS0_i",
    "_Z15uploadScaleCUDAPf",
    "_Z16copyScaleToDvicePf",
    "_Z25selectCUDAdeviceMaxMemoryv",
    "_Z32GMEMreleaseMemoryWithSupervoxelsPPfS0_S0_PPiS2_S0_PPx",
    "_Z35GMEMinitializeMemoryWithSupervoxelsPPfS_S0_S_S_xS0_PPiS2_tS0_S_PPxS3_",
    "_Z43GMEMvariationalInferenceCUDAWithSupervoxelsPfS_S_S_PiS0_S_PxP24GaussianMixtureModelCUDAxitidiibNSt7__cxx11"
    "12basic_stringIcSt11char_traitsIcESaIcEEE",
    "_ZN24GaussianMixtureModelCUDA8writeXMLERSoi",
    "_Z24calculateLocalLikelihoodRSt6vectorIdSaIdEERKS_IS_IiSaIiEESaIS4_EEPfS9_S9_PiP24GaussianMixtureModelCUDAPxxii",
    "_ZN34regularizePrecisionMatrixConstants9lambdaMinE",
    "_ZN34regularizePrecisionMatrixConstants9lambdaMaxE",
    "_ZN34regularizePrecisionMatrixConstants15maxExcentricityE",
]


def declared_c_functions():
    names = set()
    for h in ("tgmm_gmem.h", "tgmm_serve.h"):
        src = open(os.path.join(INC, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(tgmm_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_loads_without_gpu():
    lib = L.gmem()
    assert lib.tgmm_version().startswith(b"tgmm_b200")


@pytest.mark.parametrize("name", declared_c_functions())
def test_every_declared_c_function_is_exported(name):
    assert hasattr(L.gmem(), name), name
    assert name in L.GMEM_FUNCS, f"{name} has no ctypes binding"


@pytest.mark.parametrize("sym", LEGACY_SYMBOLS)
def test_reference_cpp_entry_points_exported(sym):
    out = subprocess.run(["nm", "-D", "--defined-only", L.GMEM_SO], capture_output=True, text=True).stdout
    assert sym in out.split(), sym


def test_record_layout_matches_reference():
    assert C.sizeof(L.TgmmGaussian) == 288
    offs = {"beta_k": 0, "m_k": 24, "W_k": 48, "expectedLogDetCovarianceCUDA": 96, "beta_o": 120, "m_o": 144,
            "W_o": 168, "fixed": 216, "supervoxelIdx": 220, "supervoxelNum": 284}
    for k, v in offs.items():
        assert getattr(L.TgmmGaussian, k).offset == v, k
    assert L.GAUSS_DTYPE.itemsize == 288
    assert L.GAUSS_DTYPE.fields["supervoxelNum"][1] == 284


def test_default_params_are_the_reference_defaults():
    p = L.default_params()
    assert p.max_iter_em == 400 and p.tol_likelihood == 1e-6 and p.w4dof == 1
    assert (p.lambda_min, p.lambda_max, p.max_excentricity) == (0.02, 0.2222, 9.0)
    assert p.ll_mode == L.TGMM_LL_AS_REFERENCE
    # the Python defaults (set without loading the engine) are the library's, byte for byte
    c = L.TgmmEmParams()
    L.gmem().tgmm_default_params(C.byref(c))
    assert bytes(p) == bytes(c)


def test_device_flag_bits_are_the_headers():
    src = open(os.path.join(INC, "tgmm_gmem.h")).read()
    bits = dict((k, int(v)) for k, v in re.findall(r"#define (TGMM_FLAG_[A-Z_]+) (\d+)", src))
    assert len(bits) == 7
    for k, v in bits.items():
        assert getattr(L, k) == v, k


def test_plan_bytes_is_monotone():
    def b(n, s, k, f=1):
        d = L.TgmmPlanDesc()
        d.max_vox, d.max_sv, d.max_gauss, d.max_frames, d.device = n, s, k, f, 0
        return L.gmem().tgmm_plan_bytes(C.byref(d))
    assert 0 < b(1000, 10, 10) < b(1000, 100, 100) < b(1000, 100, 100, 8)
    assert b(1000, 10, 0) == -1


def test_assign_supervoxels_matches_oracle():
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    S, K = 300, 40
    rnk = rng.dirichlet(np.ones(5) * 0.3, size=S).T.astype(np.float32).reshape(-1)
    ind = rng.integers(0, K, size=5 * S).astype(np.int32)
    g = np.zeros(K, L.GAUSS_DTYPE)
    g["supervoxelNum"] = 7  # overwritten
    got = g.copy()
    L.check(L.gmem().tgmm_assign_supervoxels(rnk.ctypes.data, ind.ctypes.data, S, got.ctypes.data, K), "assign")
    want = g.copy()
    O.lib().or_assign_supervoxels.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    O.lib().or_assign_supervoxels(rnk.ctypes.data, ind.ctypes.data, S, want.ctypes.data, K)
    np.testing.assert_array_equal(got["supervoxelNum"], want["supervoxelNum"])
    for k in range(K):
        n = want["supervoxelNum"][k]
        np.testing.assert_array_equal(got["supervoxelIdx"][k][:n], want["supervoxelIdx"][k][:n])
    assert (got["supervoxelNum"] <= 16).all()


def test_rnk_file_is_the_reference_dump_format(tmp_path):
    S = 37
    rnk = np.linspace(0, 1, 5 * S).astype(np.float32)
    ind = np.arange(5 * S, dtype=np.int32)
    p = str(tmp_path / "rnk.bin")
    L.check(L.gmem().tgmm_write_rnk_file(p.encode(), rnk.ctypes.data, ind.ctypes.data, S), "write")
    raw = open(p, "rb").read()
    hdr = np.frombuffer(raw[:8], np.int32)
    assert tuple(hdr) == (S, 5)
    np.testing.assert_array_equal(np.frombuffer(raw[8:8 + 20 * S], np.float32), rnk)
    np.testing.assert_array_equal(np.frombuffer(raw[8 + 20 * S:], np.int32), ind)


def test_host_functions_reject_bad_arguments():
    lib = L.gmem()
    assert lib.tgmm_assign_supervoxels(None, None, 3, None, 3) == L.TGMM_ERR_INVALID_ARG
    assert lib.tgmm_write_rnk_file(None, None, None, 1) == L.TGMM_ERR_INVALID_ARG
    assert b"tgmm_write_rnk_file" in lib.tgmm_last_error()


def test_legacy_header_compiles_and_links(tmp_path):
    """A C++ program written against the reference's interface builds against the library."""
    src = tmp_path / "use_legacy.cpp"
    src.write_text(open(os.path.join(ROOT, "tests", "legacy_harness.cpp")).read())
    exe = tmp_path / "use_legacy"
    r = subprocess.run(["g++", "-std=c++17", "-O1", str(src), "-I" + INC, "-I/usr/local/cuda/include",
                        L.GMEM_SO, "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + os.path.dirname(L.GMEM_SO),
                        "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_server_arena_selftest_passes_on_cpu():
    assert L.gmem().tgmm_server_selftest() == 0


def test_serve_structs_match_the_c_header(tmp_path):
    """ctypes mirrors of the serve structs have the C compiler's sizes and offsets."""
    structs = {"TgmmServerDesc": L.TgmmServerDesc, "TgmmServeRequest": L.TgmmServeRequest,
               "TgmmServeResult": L.TgmmServeResult, "TgmmServerStats": L.TgmmServerStats,
               "TgmmEmParams": L.TgmmEmParams, "TgmmEmStats": L.TgmmEmStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tgmm_serve.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", str(src), "-I" + INC, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, f"{name}.{f}"


def test_lineage_shard_covers_every_lineage_once():
    from tgmm_b200.serve import lineage_shard
    for n, w in [(4, 1), (4, 2), (7, 3), (2, 4)]:
        parts = [lineage_shard(n, r, w) for r in range(w)]
        flat = sorted(x for p in parts for x in p)
        assert flat == list(range(n))
        assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_width_setter_refuses_bad_arguments_without_a_gpu():
    lib = L.gmem()
    assert lib.tgmm_plan_set_knn_group(None, 8) == L.TGMM_ERR_INVALID_ARG
    assert lib.tgmm_plan_autotune(None, 1, None, None, None, None, None, 1, None, None) == L.TGMM_ERR_INVALID_ARG
    assert lib.tgmm_plan_set_knn_fusion(None, 1) == L.TGMM_ERR_INVALID_ARG
    assert lib.tgmm_plan_tuning(None, None, None) == L.TGMM_ERR_INVALID_ARG
    assert lib.tgmm_plan_set_stage_wait(None, 1000) == L.TGMM_ERR_INVALID_ARG


def test_gmm_xml_document_parses_and_carries_each_gaussian(tmp_path):
    """The GMM XML writer (the reference's writeXML format) needs no GPU: a document with one
    element per Gaussian, ids in order, means and precision matrices as written."""
    import xml.etree.ElementTree as ET
    import _fixtures as F
    g = np.ascontiguousarray(F.frame("hard").gauss)
    path = tmp_path / "gmm.xml"
    assert L.gmem().tgmm_write_gmm_xml(str(path).encode(), g.ctypes.data, g.shape[0]) == L.TGMM_OK
    root = ET.parse(path).getroot()
    els = root.findall("GaussianMixtureModel")
    assert len(els) == g.shape[0]
    for i, e in enumerate(els):
        assert int(e.get("id")) == i
        m = [float(v) for v in e.get("m").split()]
        np.testing.assert_allclose(m, g["m_k"][i], rtol=1e-5, atol=1e-5)
        W = np.array([float(v) for v in e.get("W").split()]).reshape(3, 3)
        np.testing.assert_allclose(W, W.T)
        np.testing.assert_allclose(W[0], g["W_k"][i][[0, 1, 2]], rtol=1e-5, atol=1e-12)
    assert L.gmem().tgmm_write_gmm_xml(None, g.ctypes.data, 1) == L.TGMM_ERR_INVALID_ARG


def test_frame_build_usage_compiles_and_links(tmp_path):
    """The C usage of the frame preparation documented for integrators compiles against the
    header and links against the library."""
    src = tmp_path / "use_frame_build.c"
    src.write_text(r'''
#include <stdio.h>
#include "tgmm_gmem.h"
int prepare(const uint16_t* raw_dev, const uint32_t* label_dev, int32_t X, int32_t Y, int32_t Z,
            int32_t n_labels, void* ws_dev, int64_t ws, float* query_dev, float* img_dev, float* cent_dev,
            int64_t* lptr_dev, uint16_t* thr_dev, int64_t max_vox, int32_t max_sv, int32_t K, void* stream,
            TgmmFrame* out) {
  TgmmFrameBuildParams fp;
  tgmm_frame_build_default_params(&fp);
  int32_t dims[3] = {X, Y, Z};
  if (ws < tgmm_frame_build_bytes(dims, n_labels)) return TGMM_ERR_BAD_SIZE;
  int64_t n_vox;
  int32_t n_sv;
  int rc = tgmm_frame_build(raw_dev, label_dev, dims, n_labels, &fp, ws_dev, ws, query_dev, img_dev, cent_dev,
                            lptr_dev, thr_dev, max_vox, max_sv, &n_vox, &n_sv, stream);
  if (rc != TGMM_OK) {
    fprintf(stderr, "%s\n", tgmm_last_error());
    return rc;
  }
  TgmmFrame f = {query_dev, img_dev, cent_dev, lptr_dev, n_vox, n_sv, K};
  *out = f;
  return TGMM_OK;
}
int main(void) { return 0; }
''')
    exe = tmp_path / "use_frame_build"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", str(src), "-I" + INC, L.GMEM_SO,
                        "-Wl,-rpath," + os.path.dirname(L.GMEM_SO), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
