"""A batch of independent molecules spread over the ranks of a process group.

One process per GPU, each with its own batched device engine: the molecules are split
by `pm7_batch_partition` (longest-processing-time by estimated cost, the same split on
every rank since it is deterministic), each rank solves its share with
`pm7_run_batch` on its own device, and the results are gathered on the host. No
collective touches the solve itself; the only exchange is the host-side gather of
the finished result dicts. The reference has no multi-device path: its callers loop
over `run_pm7` (pm7-rs src/python.rs:437, src/bin/pm7_rs.rs:176).
"""
import torch.distributed as dist

from . import api


def shard_of(molecules, rank, world, method=0):
    """Indices of the molecules `rank` solves when `world` ranks share the batch."""
    owner, _ = api.batch_partition(molecules, world, method)
    return [i for i in range(len(molecules)) if owner[i] == rank]


def run_sharded(molecules, options=None, group=None, solve=None, **common):
    """Solve `molecules` (list of (z, xyz_bohr)) across the ranks of `group`.

    Every rank calls this with the same molecules and options and gets back the full
    list of results in input order (result dict or `Pm7Error`, as `api.run_batch`).
    `solve` replaces `api.run_batch` as the per-rank solver (same signature); the
    process group may be gloo or NCCL: the gather is of host objects.
    """
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    method = int(common.get("method", 0))
    if options:
        method = int(options[0].get("method", method))
    mine = shard_of(molecules, rank, world, method)
    solver = solve or api.run_batch
    sub_opts = [options[i] for i in mine] if options is not None else None
    res = solver([molecules[i] for i in mine], options=sub_opts, **common) if mine else []
    part = list(zip(mine, res))
    if world == 1:
        parts = [part]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, part, group=group)
    out = [None] * len(molecules)
    for p in parts:
        for i, r in p:
            out[i] = r
    return out
