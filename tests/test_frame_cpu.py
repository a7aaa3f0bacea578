"""Frame preparation without a GPU: the oracle's restatement of the tracking program's input
build (trimming, size filter, erase order, centroids, background subtraction, rescale, SoA
arrays) checked against the reference's own trimSupervoxel / weightedGaussianStatistics and
eraseSupervoxelFromCurrentSegmentation compiled from their sources, the device's closed form
of the erase order checked against the reference's swap loop, and the C ABI's argument
checks."""
import ctypes as C

import numpy as np
import pytest

import _volumes as V
from oracle import oracle as O
from tgmm_b200 import _lib as L

CASES = [
    dict(seed=1),
    dict(seed=2, conn=26),
    dict(seed=3, max_size=60),            # the size rank sets the threshold
    dict(seed=4, max_pct=0.15, conn=8),   # the percentile sets it
    dict(seed=5, conn=4, min_size=20),
    dict(seed=6, conn=74, max_size=200),
    dict(seed=15, big=True, dims=(160, 144, 40), n_nuclei=80),  # a supervoxel of 67,200 voxels
]


def _coords(lin, X, Y):
    lin = lin.astype(np.int64)
    return np.stack([lin % X, (lin // X) % Y, lin // (X * Y)]).astype(np.float32)


@pytest.mark.skipif(not O.ref_f1_available(), reason="reference trimming harness not built")
@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_oracle_matches_reference_trimming_and_centroids(case):
    c = dict(max_size=3000, max_pct=0.4, conn=6, min_size=50)
    c.update({k: case[k] for k in c if k in case})
    raw, lab, n = V.make(seed=case["seed"], **{k: case[k] for k in ("dims", "n_nuclei", "big") if k in case})
    Z, Y, X = raw.shape
    rc, o = O.frame_build(raw, lab, n, O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"]))
    assert rc == 0
    ptr, lin = O.supervoxel_lists(lab, n)
    r = O.ref_trim_stats(raw, ptr, lin, c["max_size"], c["max_pct"], c["conn"])
    erased = (r["cnt"] < c["min_size"]).astype(np.uint8)
    assert erased.any() and not erased.all()
    order = O.ref_erase_order(erased)  # the reference's own erase
    N, S = o["n_vox"], o["n_sv"]
    assert S == len(order) and N == int(sum(r["cnt"][s] for s in order))
    q = o["query"].reshape(3, N)
    cent = o["cent"].reshape(3, S)
    for p, s in enumerate(order):
        a, b = o["lptr"][p], o["lptr"][p + 1]
        assert o["thr"][p] == r["thr"][s]
        assert b - a == r["cnt"][s]
        np.testing.assert_array_equal(q[:, a:b], _coords(r["lists"][s], X, Y))
        np.testing.assert_array_equal(cent[:, p].view(np.uint32), r["cent"][s].view(np.uint32))


def test_oracle_rescale_and_background():
    """img is the kept voxels' raw - thr, with every other voxel 0, rescaled to [0,1] as mylib's
    Scale_Array_To_Range does: (float)(f * (v + shift)), f = 1 / (max - min), shift = -min."""
    raw, lab, n = V.make(seed=7)
    Z, Y, X = raw.shape
    rc, o = O.frame_build(raw, lab, n)
    assert rc == 0
    N = o["n_vox"]
    q = o["query"].reshape(3, N).astype(np.int64)
    lin = q[0] + X * (q[1] + Y * q[2])
    thr = np.repeat(o["thr"].astype(np.int64), np.diff(o["lptr"]))
    sub = (raw.reshape(-1)[lin].astype(np.int64) - thr) & 0xFFFF
    assert (sub > 0).all()
    f = 1.0 / float(sub.max())
    np.testing.assert_array_equal(o["img"], (f * (sub.astype(np.float32).astype(np.float64) + 0.0)).astype(np.float32))
    assert o["img"].max() == 1.0 and o["img"].min() > 0


def _closed_form(erased):
    """The device's erase order: output p is p when kept, else the end of the chain from
    n-m+rank(p), each erased tail position q stepping to n-m+rank(q)."""
    e = np.asarray(erased, bool)
    n, m = len(e), int(e.sum())
    S = n - m
    rank = np.concatenate([[0], np.cumsum(e)[:-1]])
    nxt = np.arange(n)
    nxt[S:] = np.where(e[S:], S + rank[S:], np.arange(S, n))
    for _ in range(64):  # pointer jumping
        nxt[S:] = nxt[nxt[S:]]
    return np.array([nxt[S + rank[p]] if e[p] else p for p in range(S)], np.int32)


@pytest.mark.parametrize("seed", range(12))
def test_erase_order_closed_form_is_the_reference_swap_loop(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 400))
    erased = rng.random(n) < rng.choice([0.05, 0.3, 0.7, 0.95])
    if erased.all():
        erased[rng.integers(0, n)] = False
    np.testing.assert_array_equal(_closed_form(erased), O.erase_order(erased.astype(np.uint8)))


@pytest.mark.skipif(not O.ref_f1_available(), reason="reference trimming harness not built")
@pytest.mark.parametrize("seed", range(8))
def test_erase_order_is_the_references(seed):
    """The oracle's restatement and the device's closed form against the reference's own
    hierarchicalSegmentation::eraseSupervoxelFromCurrentSegmentation."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 3000))
    erased = (rng.random(n) < rng.choice([0.02, 0.2, 0.5, 0.9])).astype(np.uint8)
    if erased.all():
        erased[0] = 0
    ref = O.ref_erase_order(erased)
    np.testing.assert_array_equal(O.erase_order(erased), ref)
    np.testing.assert_array_equal(_closed_form(erased.astype(bool)), ref)


def test_erase_order_examples():
    # erase {1, 3} of 5: 3 trades with 4, then 1 with the new last (the old 4)
    np.testing.assert_array_equal(O.erase_order(np.array([0, 1, 0, 1, 0], np.uint8)), [0, 4, 2])
    np.testing.assert_array_equal(O.erase_order(np.array([0, 1, 0, 0, 1], np.uint8)), [0, 3, 2])


def test_oracle_reports_errors_like_the_reference():
    raw, lab, n = V.make(seed=8, n_nuclei=4)
    assert O.frame_build(raw, lab, n, O.frame_params(min_size=10 ** 6))[0] == 5  # every supervoxel erased
    bad = lab.copy()
    bad[0, 0, 0] = n + 1
    assert O.frame_build(raw, bad, n)[0] == 1
    assert O.frame_build(raw, lab, n, O.frame_params(conn=75))[0] == 1


def test_otsu_threshold_cases():
    lib = O.lib()
    lib.or_otsu.argtypes = [C.c_void_p, C.c_int32]
    lib.or_otsu.restype = C.c_float
    flat = np.full(10, 7.0, np.float32)
    assert lib.or_otsu(flat.ctypes.data, 10) == -np.finfo(np.float32).max
    two = np.array([10.0] * 5 + [200.0] * 5, np.float32)
    t = lib.or_otsu(two.ctypes.data, 10)
    assert 10.0 <= t < 200.0


def _without_a_device(body):
    """Runs body (a function of this module) in a child process that sees no CUDA device,
    so that a host check dropped or reordered shows up as a CUDA error on the host instead
    of a kernel launched on the made-up addresses these tests pass."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    code = f"import sys; sys.path[:0] = [{here!r}, {os.path.dirname(here)!r}]; import test_frame_cpu as t; t.{body}()"
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_abi_frame_build_checks_arguments_without_a_gpu():
    _without_a_device("_check_frame_build_arguments")


def _check_frame_build_arguments():
    lib = L.gmem()
    dims = (C.c_int32 * 3)(64, 48, 16)
    assert lib.tgmm_frame_build_bytes(dims, 0) == -1
    b1, b2 = lib.tgmm_frame_build_bytes(dims, 10), lib.tgmm_frame_build_bytes(dims, 1000)
    assert 0 < b1 < b2
    assert b1 >= 10 * 64 * 48 * 16  # lists, values, queues, flood bits
    p = L.TgmmFrameBuildParams()
    lib.tgmm_frame_build_default_params(C.byref(p))
    assert (p.max_nuclei_size, round(p.max_percentile, 6), p.conn3d, p.min_nuclei_size) == (3000, 0.4, 6, 50)
    nv, ns = C.c_int64(0), C.c_int32(0)
    rc = lib.tgmm_frame_build(None, None, dims, 10, C.byref(p), None, 0, None, None, None, None, None, 0, 0,
                              C.byref(nv), C.byref(ns), None)
    assert rc == L.TGMM_ERR_INVALID_ARG
    fake = C.c_void_p(256)  # never dereferenced: the checks below fail first
    p.conn3d = 75
    rc = lib.tgmm_frame_build(fake, fake, dims, 10, C.byref(p), fake, b1, fake, fake, fake, fake, None, 1, 1,
                              C.byref(nv), C.byref(ns), None)
    assert rc == L.TGMM_ERR_INVALID_ARG and b"conn3d" in lib.tgmm_last_error()
    p.conn3d = 6
    rc = lib.tgmm_frame_build(fake, fake, dims, 10, C.byref(p), fake, b1 - 1, fake, fake, fake, fake, None, 1, 1,
                              C.byref(nv), C.byref(ns), None)
    assert rc == L.TGMM_ERR_BAD_SIZE


def test_bench_frames_reference_arm_runs_on_cpu():
    """bench.py --impl reference --workload frames: the host build's restatement on a small
    synthetic volume prints one JSON line of the frames metric (no GPU)."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload", "frames",
                        "--fb-dims", "256,128,32", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "frame preparations/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == ("reference" if O.ref_f1_available() else "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["n_sv_out"] > 0


@pytest.mark.skipif(not O.ref_f1_available(), reason="reference trimming harness not built")
@pytest.mark.parametrize("seed", range(10))
def test_trimming_matches_reference_on_random_volumes(seed):
    """Random small volumes and parameters: every supervoxel's threshold, kept voxels and
    centroid from the oracle equal the reference's own, through the whole frame build."""
    rng = np.random.default_rng(1000 + seed)
    dims = (int(rng.integers(40, 90)), int(rng.integers(30, 70)), int(rng.integers(8, 20)))
    raw, lab, n = V.make(dims=dims, n_nuclei=int(rng.integers(5, 25)), seed=2000 + seed,
                         background=float(rng.uniform(50, 300)))
    c = dict(max_size=int(rng.choice([40, 150, 3000])), max_pct=float(rng.choice([0.1, 0.4, 0.75])),
             conn=int(rng.choice([4, 6, 8, 26, 74])), min_size=int(rng.choice([1, 20, 50])))
    rc, o = O.frame_build(raw, lab, n, O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"]))
    ptr, lin = O.supervoxel_lists(lab, n)
    r = O.ref_trim_stats(raw, ptr, lin, c["max_size"], c["max_pct"], c["conn"])
    erased = (r["cnt"] < c["min_size"]).astype(np.uint8)
    if erased.all():
        assert rc == 5
        return
    assert rc == 0
    order = O.ref_erase_order(erased)
    Z, Y, X = raw.shape
    N, S = o["n_vox"], o["n_sv"]
    assert S == len(order)
    q = o["query"].reshape(3, N)
    for p, s in enumerate(order):
        a, b = o["lptr"][p], o["lptr"][p + 1]
        assert o["thr"][p] == r["thr"][s] and b - a == r["cnt"][s]
        np.testing.assert_array_equal(q[:, a:b], _coords(r["lists"][s], X, Y))
        np.testing.assert_array_equal(o["cent"].reshape(3, S)[:, p].view(np.uint32), r["cent"][s].view(np.uint32))


@pytest.mark.parametrize("name", ["frame_default", "frame_conn26", "frame_big"])
def test_oracle_matches_committed_reference_outputs(name):
    """The committed outputs of the reference's own trimming, statistics and erase
    (tests/golden/make_frame_golden.py) against the oracle's frame build: needs neither the
    reference sources nor a GPU."""
    import os
    import sys
    gold_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, gold_dir)
    import make_frame_golden as MG
    with np.load(os.path.join(gold_dir, f"{name}.npz")) as z:
        g = {k: z[k] for k in z.files}
    c = MG.FRAME_CASES[name]
    raw, lab, n = MG.volume(c)
    assert MG.digest(raw, lab) == str(g["input_sha256"]), "the volume generator changed: regenerate the fixtures"
    rc, o = O.frame_build(raw, lab, n, O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"]))
    assert rc == 0
    Z, Y, X = raw.shape
    order = g["order"]
    N, S = o["n_vox"], o["n_sv"]
    assert S == len(order) and N == int(g["cnt"][order].sum())
    q = o["query"].reshape(3, N)
    for p, s in enumerate(order):
        a, b = o["lptr"][p], o["lptr"][p + 1]
        assert o["thr"][p] == g["thr"][s] and b - a == g["cnt"][s]
        np.testing.assert_array_equal(q[:, a:b], _coords(g["kept_lin"][g["kept_ptr"][s]:g["kept_ptr"][s + 1]], X, Y))
        np.testing.assert_array_equal(o["cent"].reshape(3, S)[:, p].view(np.uint32), g["cent"][s].view(np.uint32))


@pytest.mark.skipif(not O.ref_f1_available(), reason="reference trimming harness not built")
@pytest.mark.parametrize("case", CASES + [dict(seed=7), dict(seed=8, n_nuclei=6, min_size=120)],
                         ids=[str(c) for c in CASES] + ["seed7", "seed8-min120"])
def test_oracle_frame_build_is_the_reference_host_build(case):
    """The whole build, bit for bit: the oracle against main's loop run with the reference's own
    trimming, statistics and erase (coordinates, rescaled intensities, centroids, CSR)."""
    c = dict(max_size=3000, max_pct=0.4, conn=6, min_size=50)
    c.update({k: case[k] for k in c if k in case})
    raw, lab, n = V.make(seed=case["seed"], **{k: case[k] for k in ("dims", "n_nuclei", "big") if k in case})
    p = O.frame_params(c["max_size"], c["max_pct"], c["conn"], c["min_size"])
    rc, o = O.frame_build(raw, lab, n, p)
    rr, r = O.ref_frame_build(raw, lab, n, p)
    assert rc == rr
    if rc:
        return
    assert (o["n_vox"], o["n_sv"]) == (r["n_vox"], r["n_sv"])
    for k in ("query", "img", "cent", "lptr"):
        np.testing.assert_array_equal(o[k].view(np.uint8), r[k].view(np.uint8), err_msg=k)


def test_abi_frame_build_refuses_bad_sizes_and_parameters_without_a_gpu():
    """Every argument check of tgmm_frame_build happens on the host before any device work."""
    _without_a_device("_check_frame_build_refusals")


def _check_frame_build_refusals():
    lib = L.gmem()
    p = L.TgmmFrameBuildParams()
    lib.tgmm_frame_build_default_params(C.byref(p))
    nv, ns = C.c_int64(0), C.c_int32(0)
    fake = C.c_void_p(4096)  # never dereferenced: each call below is refused first
    ws = 1 << 40

    def call(dims, n=10, label=fake, params=p, max_vox=1, max_sv=1):
        d = (C.c_int32 * 3)(*dims)
        return lib.tgmm_frame_build(fake, label, d, n, C.byref(params), fake, ws, fake, fake, fake, fake, None,
                                    max_vox, max_sv, C.byref(nv), C.byref(ns), None)

    assert call((0, 4, 4)) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), n=0) == L.TGMM_ERR_INVALID_ARG
    assert call((4096, 4096, 256)) == L.TGMM_ERR_BAD_SIZE            # 2^32 voxels
    assert call((4, 4, 4), n=(1 << 24) + 1) == L.TGMM_ERR_BAD_SIZE
    assert call((4, 4, 4), label=C.c_void_p(4100)) == L.TGMM_ERR_INVALID_ARG  # label not 16-byte aligned
    assert b"aligned" in lib.tgmm_last_error()
    bad = L.TgmmFrameBuildParams(p.max_nuclei_size, 1.5, p.conn3d, p.min_nuclei_size)
    assert call((4, 4, 4), params=bad) == L.TGMM_ERR_INVALID_ARG
    bad = L.TgmmFrameBuildParams(-1, p.max_percentile, p.conn3d, p.min_nuclei_size)
    assert call((4, 4, 4), params=bad) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), max_vox=-1) == L.TGMM_ERR_INVALID_ARG
    ms = (C.c_float * L.TGMM_FRAME_BUILD_STAGES)()
    d = (C.c_int32 * 3)(4, 4, 4)
    assert lib.tgmm_frame_build_timed(fake, fake, d, 10, C.byref(p), fake, ws, fake, fake, fake, fake, None, 1, 1,
                                      C.byref(nv), C.byref(ns), None, None) == L.TGMM_ERR_INVALID_ARG


def test_abi_list_build_refuses_bad_arguments_without_a_gpu():
    """Every argument check of tgmm_frame_build_lists happens on the host before any device work."""
    _without_a_device("_check_list_build_refusals")


def _check_list_build_refusals():
    lib = L.gmem()
    p = L.TgmmFrameBuildParams()
    lib.tgmm_frame_build_default_params(C.byref(p))
    nv, ns = C.c_int64(0), C.c_int32(0)
    fake = C.c_void_p(4096)  # never dereferenced: each call below is refused first
    ws = 1 << 40
    ms = (C.c_float * L.TGMM_FRAME_BUILD_STAGES)()

    def call(dims, n=10, n_list=50, lin=fake, ptr=fake, params=p, max_vox=1, max_sv=1, wsb=ws):
        d = (C.c_int32 * 3)(*dims)
        return lib.tgmm_frame_build_lists(lin, fake, ptr, n_list, d, n, C.byref(params), fake, wsb, fake, fake, fake,
                                          fake, None, max_vox, max_sv, C.byref(nv), C.byref(ns), None, ms)

    assert call((0, 4, 4)) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), n=0) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), n_list=-1) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), lin=None) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), ptr=None) == L.TGMM_ERR_INVALID_ARG
    assert call((4096, 4096, 256)) == L.TGMM_ERR_BAD_SIZE            # 2^32 voxels
    assert call((4, 4, 4), n_list=65) == L.TGMM_ERR_BAD_SIZE          # more entries than voxels
    assert call((4, 4, 4), n=(1 << 24) + 1) == L.TGMM_ERR_BAD_SIZE
    bad = L.TgmmFrameBuildParams(p.max_nuclei_size, 1.5, p.conn3d, p.min_nuclei_size)
    assert call((4, 4, 4), params=bad) == L.TGMM_ERR_INVALID_ARG
    bad = L.TgmmFrameBuildParams(p.max_nuclei_size, p.max_percentile, 5, p.min_nuclei_size)
    assert call((4, 4, 4), params=bad) == L.TGMM_ERR_INVALID_ARG
    assert call((4, 4, 4), max_sv=-1) == L.TGMM_ERR_INVALID_ARG
    need = lib.tgmm_frame_build_lists_bytes((C.c_int32 * 3)(4, 4, 4), 10, 50)
    assert need > 0
    assert call((4, 4, 4), n_list=50, wsb=need - 1) == L.TGMM_ERR_BAD_SIZE
    assert b"workspace" in lib.tgmm_last_error()
    assert lib.tgmm_frame_build_lists_bytes((C.c_int32 * 3)(4, 4, 4), 10, -1) == -1
