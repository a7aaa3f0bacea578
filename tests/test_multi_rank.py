"""Multi-process paths on CPU with the gloo backend (world size 2, rendezvous on
127.0.0.1): the whole-job reduction of bench.py (slowest rank's time, every rank's
voxels) and the lineage sharding of the served form -- each rank runs its lineages'
frames (here through the CPU oracle) and the gathered results cover every lineage once
and equal a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

WORLD = 2


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def tiny_lineages():
    from tgmm_b200 import synth
    specs = [synth.VolumeSpec(dims=(48, 48, 24), n_nuclei=6 + i, axis_min=3.0, axis_max=4.5) for i in range(3)]
    return [synth.time_series(sp, seed=300 + i, n_frames=2, divide_frac=0.1) for i, sp in enumerate(specs)]


def run_lineage(frames):
    """Frames of one lineage through the oracle, posterior -> prior between frames."""
    from oracle import oracle as O
    g = frames[0].gauss.copy()
    out = []
    for f in frames:
        o = O.em_run(f.query, f.img, f.centroids, f.label_ptr, g, O.params(max_iter=5, tol=-1.0))
        out.append((o["ind"].tobytes(), o["rnk"].tobytes(), o["gauss"]["m_k"].tobytes()))
        g = o["gauss"].copy()
        O.lib().or_update_priors(g.ctypes.data, g.shape[0], 0.01, 1.0, 0.8, float(g["alpha_k"].sum()))
    return out


def worker(rank, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    try:
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
        import bench
        from tgmm_b200.serve import lineage_shard
        value, vi, max_ms, tv = bench.reduce_job(10.0 + 5 * rank, 1000 * (rank + 1), 4, WORLD, "cpu")
        series = tiny_lineages()
        mine = {li: run_lineage(series[li]) for li in lineage_shard(len(series), rank, WORLD)}
        gathered = [None] * WORLD
        dist.all_gather_object(gathered, mine)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, dict(value=value, vi=vi, max_ms=max_ms, tv=tv, gathered=gathered)))
    except Exception as e:  # report, never hang the parent
        q.put((rank, {"error": repr(e)}))


def test_two_rank_reduction_and_lineage_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(WORLD):
        rank, res = q.get(timeout=240)
        out[rank] = res
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    for r in range(WORLD):
        assert "error" not in out[r], out[r]
        assert out[r]["max_ms"] == 15.0               # the slowest rank
        assert out[r]["tv"] == 3000.0                 # every rank's voxels
        assert out[r]["value"] == pytest.approx(WORLD * 4 / 0.015)
    merged = {}
    for part in out[0]["gathered"]:
        for li, res in part.items():
            assert li not in merged, "a lineage ran on two ranks"
            merged[li] = res
    series = tiny_lineages()
    assert sorted(merged) == list(range(len(series)))
    for li, fr in enumerate(series):
        assert merged[li] == run_lineage(fr)
