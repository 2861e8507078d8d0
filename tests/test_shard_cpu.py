"""Multi-rank fan split (infraga_b200.shard) on CPU: two gloo ranks each trace
their shard of a fan -- with the oracle standing in for the GPU fan call, so
no device is needed -- and the gathered result equals the single-rank result
row for row, in the reference's launch order (src/main.infraga.3d.mpi.cpp:
inclinations dealt round-robin over ranks, rows collected on rank 0)."""
import os
import socket
import tempfile

import numpy as np
import pytest

from infraga_b200 import shard, synth
from tests._cases import profile_path

FAN_KW = dict(bounces=2, rng_max=600.0, write_rays=0)


def _angles():
    return synth.fan_angles(2.0, 40.0, 3.0, 30.0, 120.0, 45.0)


def _oracle_runner(met, kw, th, ph):
    from oracle import oracle
    rows, steps = oracle.fan_3d(met, th, ph, **kw)
    pos = {(a, b): i for i, (a, b) in enumerate(zip(th.tolist(), ph.tolist()))}
    ray_index = np.array([pos[(r[0], r[1])] for r in rows.tolist()], dtype=np.int64)
    return {"arrivals": rows, "ray_index": ray_index, "ray_steps": steps,
            "ray_status": np.zeros(th.size, np.int32), "total_steps": int(steps.sum())}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, mode, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        th, ph = _angles()
        res = shard.fan_run_sharded(profile_path(0), FAN_KW, th, ph, mode=mode, runner=_oracle_runner)
        if rank == 0:
            np.savez(out, **res)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", shard.MODES)
def test_shards_partition_launch_list(mode):
    for n in (0, 1, 7, 71520):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_indices(n, r, world, mode) for r in range(world)]
            allidx = np.sort(np.concatenate(parts))
            assert np.array_equal(allidx, np.arange(n))
            assert max(p.size for p in parts) - min(p.size for p in parts) <= 1


def test_merge_restores_launch_order():
    # a fan whose rays have different arrival counts, dealt over three ranks
    counts = np.array([2, 0, 1, 3, 1, 2, 0])
    rows, ri = [], []
    for i, c in enumerate(counts):
        for b in range(c):
            rows.append([i, 0, b] + [float(i * 10 + b)] * 9)
            ri.append(i)
    full = {"arrivals": np.array(rows, float), "ray_index": np.array(ri), "ray_steps": counts * 100,
            "ray_status": counts % 2, "total_steps": int(counts.sum() * 100)}
    parts = []
    for r in range(3):
        idx = shard.shard_indices(counts.size, r, 3)
        sel = np.isin(full["ray_index"], idx)
        local = np.searchsorted(idx, full["ray_index"][sel])
        parts.append((idx, {"arrivals": full["arrivals"][sel], "ray_index": local, "ray_steps": full["ray_steps"][idx],
                            "ray_status": full["ray_status"][idx], "total_steps": int(full["ray_steps"][idx].sum())}))
    m = shard.merge_shards(parts[::-1], counts.size)
    assert np.array_equal(m["arrivals"], full["arrivals"])
    assert np.array_equal(m["ray_index"], full["ray_index"])
    assert np.array_equal(m["ray_steps"], full["ray_steps"])
    assert np.array_equal(m["ray_status"], full["ray_status"])
    assert m["total_steps"] == full["total_steps"]


@pytest.mark.parametrize("mode", shard.MODES)
def test_two_gloo_ranks_gather_equals_single_rank(mode):
    import torch.multiprocessing as mp
    th, ph = _angles()
    single = _oracle_runner(profile_path(0), FAN_KW, th, ph)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "rank0.npz")
        ctx = mp.get_context("spawn")
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, mode, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        got = dict(np.load(out))
    assert np.array_equal(got["arrivals"], single["arrivals"])
    assert np.array_equal(got["ray_index"], single["ray_index"])
    assert np.array_equal(got["ray_steps"], single["ray_steps"])
    assert int(got["total_steps"]) == single["total_steps"]
