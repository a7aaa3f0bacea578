"""CPU checks of the seeded workload generator: determinism, CSR validity, supervoxel
rules (contiguous ascending runs, minimum size), intensity range, centroids, Gaussians."""
import numpy as np
import pytest

import _fixtures as F
from tgmm_b200 import synth


def test_generation_is_deterministic():
    a = synth.generate(synth.TINY, seed=11)
    b = synth.generate(synth.TINY, seed=11)
    for k in ("query", "img", "centroids", "label_ptr"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k))
    np.testing.assert_array_equal(a.gauss.view(np.uint8), b.gauss.view(np.uint8))
    c = synth.generate(synth.TINY, seed=12)
    assert c.n_vox != a.n_vox or not np.array_equal(c.img, a.img)


@pytest.mark.parametrize("name", ["tiny", "small", "c1", "big"])
def test_frame_structure(name):
    f = F.frame(name)
    spec = f.spec
    lp = f.label_ptr
    assert lp[0] == 0 and lp[-1] == f.n_vox and np.all(np.diff(lp) >= spec.min_size)
    X, Y, Z = spec.dims
    q = f.query.reshape(3, -1)
    assert q.min() >= 0 and q[0].max() < X and q[1].max() < Y and q[2].max() < Z
    lin = (q[2].astype(np.int64) * Y + q[1].astype(np.int64)) * X + q[0].astype(np.int64)
    for s in range(f.n_sv):
        run = lin[lp[s]:lp[s + 1]]
        assert np.all(np.diff(run) > 0), "voxels of a supervoxel ascend in linear index"
    assert len(np.unique(lin)) == f.n_vox, "a voxel belongs to one supervoxel"
    assert f.img.min() > 0 and f.img.max() == pytest.approx(1.0)
    c = f.centroids.reshape(3, -1)
    for s in range(f.n_sv):
        w = f.img[lp[s]:lp[s + 1]].astype(np.float64)
        cen = (q[:, lp[s]:lp[s + 1]] * w).sum(1) / w.sum()
        np.testing.assert_allclose(c[:, s], cen, rtol=1e-5, atol=1e-4)


def test_c1_sizes_match_the_configuration():
    f = F.frame("c1")
    assert 60_000 < f.n_vox < 200_000  # ~110k foreground voxels
    assert 250 <= f.n_gauss <= 300 and f.n_sv >= f.n_gauss


def test_first_frame_gaussians_follow_tgmm_initialisation():
    f = F.frame("small")
    g = f.gauss
    lp = f.label_ptr
    Nk = np.zeros(f.nuclei.n)
    for s in range(f.n_sv):
        Nk[f.sv_nucleus[s]] += f.img[lp[s]:lp[s + 1]].astype(np.float64).sum()
    n = Nk[f.gauss_nucleus]
    np.testing.assert_allclose(g["alpha_k"], n, rtol=1e-12)
    np.testing.assert_allclose(g["beta_k"], n, rtol=1e-12)
    np.testing.assert_allclose(g["nu_k"], 2 * n, rtol=1e-12)   # nu *= 2 after updatePriors
    np.testing.assert_allclose(g["beta_o"], np.maximum(0.1 * n, 1e-5), rtol=1e-12)
    np.testing.assert_allclose(g["nu_o"], np.maximum(0.1 * n, 3.0), rtol=1e-12)
    np.testing.assert_allclose(g["alpha_o"], 0.1 * n, rtol=1e-12)
    np.testing.assert_allclose(g["m_o"], g["m_k"])
    assert np.abs(g["m_k"] - f.nuclei.centre[f.gauss_nucleus]).max() < 10  # jitter of 1.5 voxels
    assert (g["W_k"][:, 2] == 0).all() and (g["W_k"][:, 4] == 0).all()  # 4-DOF regularisation


def test_batch_specs_follow_the_density_rule():
    specs = synth.batch_specs(64, seed=3)
    assert len(specs) == 64
    for s in specs:
        X, Y, Z = s.dims
        assert 128 <= X <= 512 and 128 <= Y <= 512 and 64 <= Z <= 128
        assert s.n_nuclei == int(np.clip(round(X * Y * Z / 3000), 100, 5000))


def test_time_series_motion_and_division():
    rng = np.random.default_rng(0)
    nuc = synth.random_nuclei(synth.TINY, 1)
    nxt = synth.evolve_nuclei(nuc, synth.TINY, rng, divide_frac=0.5)
    assert nxt.n > nuc.n
    assert np.all(nxt.centre >= 0) and np.all(nxt.centre <= np.array(synth.TINY.dims) - 1)


def test_bench_reference_arm_never_maps_the_engine():
    """bench.py --impl reference (the reference's CPU arithmetic, each step one whole 20-iteration
    EM call) runs on the CPU and never loads the CUDA engine library: the data generator and
    the CPU arithmetic need nothing from it."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'c1', '--steps', '1', "
            "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "print('MAPPED', 'libtgmm_gmem.so' in open('/proc/self/maps').read())")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "MAPPED False"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["value"] > 0 and line["config"]["em_iterations"] == 20
    assert abs(line["ms_per_step"] - 1e3 / line["value"]) < 1e-6 * line["ms_per_step"]


def test_runs_cover_each_supervoxel_in_order():
    """synth.runs_of: each supervoxel's runs expand to its voxels' linear indices in order; runs
    never cross a supervoxel boundary and are split at max_len."""
    f = synth.generate(synth.TINY, seed=3)
    lin = f.compact()[0].astype(np.int64)
    for max_len in (65535, 5, 1):
        rp, rs, rl = synth.runs_of(lin, f.label_ptr, max_len=max_len)
        assert rp.dtype == np.int32 and rs.dtype == np.uint32 and rl.dtype == np.uint16
        assert rp[0] == 0 and rp[-1] == rs.shape[0] and rl.max() <= max_len and rl.min() >= 1
        for s in range(f.n_sv):
            a, b = f.label_ptr[s], f.label_ptr[s + 1]
            got = np.concatenate([np.arange(int(x), int(x) + int(n)) for x, n in
                                  zip(rs[rp[s]:rp[s + 1]], rl[rp[s]:rp[s + 1]])] or [np.zeros(0, np.int64)])
            np.testing.assert_array_equal(got, lin[a:b])
    # one long run, an empty supervoxel, a run cut at max_len
    rp, rs, rl = synth.runs_of(np.arange(200000), np.array([0, 150000, 150000, 200000]))
    np.testing.assert_array_equal(rp, [0, 3, 3, 4])
    np.testing.assert_array_equal(rl, [65535, 65535, 18930, 50000])
    np.testing.assert_array_equal(rs, [0, 65535, 131070, 150000])
