"""Sharding a batch over ranks (CPU: gloo, world size 2).

The batch split (`pm7_batch_partition`) is host logic and runs without a GPU; the
per-rank solver is replaced by the oracle so the whole path — split, per-rank solve,
host-side gather in input order — runs on CPU ranks. On GPUs each rank's solver is
`api.run_batch` on its own device; nothing else changes.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import harness
from pm7b200 import api, shard
from pm7b200 import geometry as G


def _small_batch():
    mols = [G.water_cluster(k, seed=k) for k in (1, 2, 3)] + [G.alkane(n, seed=n) for n in (1, 2, 3, 4)]
    mols.append((np.array([1, 1], np.uint8), np.zeros((2, 3))))  # coincident atoms: an error result
    return mols


def _oracle_batch(molecules, options=None, **common):
    out = []
    for i, (z, x) in enumerate(molecules):
        o = dict(common)
        if options is not None:
            o.update(options[i])
        try:
            out.append(harness.run(z, x, **o))
        except harness.OracleError as e:
            out.append(api.Pm7Error(e.code, str(e)))
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mols = _small_batch()
        res = shard.run_sharded(mols, solve=_oracle_batch)
        mine = shard.shard_of(mols, rank, world)
        queue.put((rank, mine, [r if isinstance(r, dict) else ("error", r.code) for r in res]))
    finally:
        dist.destroy_process_group()


def test_partition_is_balanced_and_deterministic():
    mols = G.batch(256, seed=3)
    owner, load = api.batch_partition(mols, 4)
    assert set(owner.tolist()) == {0, 1, 2, 3}
    assert load.max() / load.mean() < 1.02  # LPT on many small jobs: near-even
    owner2, _ = api.batch_partition(mols, 4)
    assert np.array_equal(owner, owner2)
    one, load1 = api.batch_partition(mols, 1)
    assert not one.any() and abs(load1[0] - load.sum()) < 1e-6 * load.sum()


def test_partition_puts_the_heaviest_molecules_apart():
    mols = [G.water_cluster(k, seed=k) for k in (60, 55, 2, 2, 2, 2)]
    owner, _ = api.batch_partition(mols, 2)
    assert owner[0] != owner[1]


def test_partition_rejects_bad_arguments():
    with pytest.raises(api.Pm7Error) as info:
        api.batch_partition(_small_batch(), 0)
    assert info.value.code == 1


def test_sharded_batch_on_two_gloo_ranks_matches_one_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, mine, res = queue.get(timeout=300)
        got[rank] = (mine, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mols = _small_batch()
    # the ranks split the batch into disjoint shares that cover it
    shares = sorted(i for r in got for i in got[r][0])
    assert shares == list(range(len(mols))) and got[0][0] and got[1][0]
    direct = _oracle_batch(mols)
    for rank in got:
        res = got[rank][1]
        for r, d in zip(res, direct):
            if isinstance(d, api.Pm7Error):
                assert r == ("error", d.code)
            else:
                assert r["heat_of_formation_kcal"] == d["heat_of_formation_kcal"]
                assert np.array_equal(r["charges"], d["charges"])
