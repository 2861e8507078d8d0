"""Ray fans split over ranks (one process per GPU) and gathered in the
reference's order.

The reference's MPI build (src/main.infraga.3d.mpi.cpp) deals the
inclinations of each azimuth round-robin over the ranks (rank r traces
theta_min + (i * world + r) * theta_step, :370-371) and sends every result row
to rank 0, which writes them in launch order (:431-433 and the arrival block
after it).  Rays are independent, so the split needs no exchange while the
rays run: here each rank traces its shard of the fan's launch list with one
fan call on its own GPU, and one gather at the end brings the rows to the
destination rank, which orders them by launch index -- the order the serial
reference and a single-rank fan produce.

``interleave`` (the default) deals the launch list round-robin like the
reference, which balances ranks when ray lengths vary smoothly with
inclination; ``contiguous`` gives each rank one block of the list.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

MODES = ("interleave", "contiguous")


def shard_indices(n_rays: int, rank: int, world: int, mode: str = "interleave") -> np.ndarray:
    """Launch indices (into the fan's theta/phi lists) that ``rank`` of
    ``world`` traces.  Every index belongs to exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    if mode == "interleave":
        return np.arange(rank, n_rays, world, dtype=np.int64)
    if mode == "contiguous":
        lo = (n_rays * rank) // world
        hi = (n_rays * (rank + 1)) // world
        return np.arange(lo, hi, dtype=np.int64)
    raise ValueError(f"unknown shard mode {mode!r} (one of {MODES})")


def merge_shards(parts, n_rays: int) -> dict:
    """Merge per-rank results ``(indices, result)`` into one fan result in
    launch order: arrivals grouped by ray (launch index ascending) with each
    ray's bounces in order, per-ray steps and status at their launch index."""
    rows, ray_index, steps, status = [], [], np.zeros(n_rays, np.int64), np.zeros(n_rays, np.int32)
    total = 0
    for idx, r in parts:
        idx = np.asarray(idx, dtype=np.int64)
        rows.append(np.asarray(r["arrivals"], dtype=np.float64).reshape(-1, 12))
        ray_index.append(idx[np.asarray(r["ray_index"], dtype=np.int64)])
        steps[idx] = r["ray_steps"]
        if "ray_status" in r:
            status[idx] = r["ray_status"]
        total += int(r["total_steps"])
    arr = np.concatenate(rows) if rows else np.zeros((0, 12))
    ri = np.concatenate(ray_index) if ray_index else np.zeros(0, np.int64)
    order = np.argsort(ri, kind="stable")   # stable: a ray's arrivals keep their bounce order
    return {"arrivals": arr[order], "ray_index": ri[order].astype(np.int32), "ray_steps": steps,
            "ray_status": status, "total_steps": total}


def fan_run_sharded(atmo, params, theta_deg, phi_deg, group=None, dst: int = 0, mode: str = "interleave",
                    runner: Callable | None = None):
    """Trace one fan over all ranks of ``group`` (torch.distributed, already
    initialised; nccl or gloo) and gather the result on rank ``dst``.

    Every rank passes the whole launch list; each traces its shard with
    ``runner(atmo, params, theta, phi)`` (default: :func:`infraga_b200.fan_run`
    on the rank's current GPU) and rank ``dst`` returns the merged result in
    launch order (the dict of ``fan_run``); the other ranks return None."""
    import torch.distributed as dist
    if runner is None:
        from ._lib import fan_run as runner
    th = np.ascontiguousarray(theta_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
    if th.shape != ph.shape:
        raise ValueError("theta and phi lists differ in length")
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    idx = shard_indices(th.size, rank, world, mode)
    r = runner(atmo, params, th[idx], ph[idx])
    mine = (idx, {k: r[k] for k in ("arrivals", "ray_index", "ray_steps", "ray_status", "total_steps") if k in r})
    dst_global = dist.get_global_rank(group, dst) if group is not None else dst
    gathered = [None] * world if rank == dst else None
    dist.gather_object(mine, gathered, dst=dst_global, group=group)
    if rank != dst:
        return None
    return merge_shards(gathered, th.size)
