"""Failure paths on the device, exercised without faulting or hanging the GPU.

* Bounded waits: the tcgen05 squaring's mbarrier waits have a time limit. The drill entry
  point withholds every copy of the pipeline (a phase that nothing completes), so each wait
  runs out; the kernel must return, report PM7_ERR_TIMEOUT, and leave the context usable.
* Admission by HBM footprint (the serving engine's version of the reference's memory guard,
  src/memory.rs:95-118): with a budget that holds only a few requests, the others wait,
  every request finishes, and each result equals the one the request gets alone.
* The multi-GPU shard path (`shard.run_sharded`) through the real `pm7_run_batch` on one
  rank.
"""
import math
import time

import numpy as np
import pytest

from oracle import harness
from pm7b200 import api, shard
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu

PM7_ERR_TIMEOUT = 10


def test_expired_pipeline_waits_report_timeout_and_the_context_survives():
    t = time.perf_counter()
    assert api.tf32_wait_drill(128) == PM7_ERR_TIMEOUT
    assert time.perf_counter() - t < 30.0
    assert api.tf32_wait_drill(300) == PM7_ERR_TIMEOUT  # several CTAs, each gives up on its own
    # the same kernel with its copies in place, then a whole solve, on the same context
    rng = np.random.default_rng(1)
    a = rng.standard_normal((200, 200))
    x = (a + a.T) / 2
    c = api.square_tf32(x)
    assert np.max(np.abs(c - x @ x)) < 1e-4 * np.max(np.abs(x @ x))
    z, xyz = G.decane(0)
    r = api.run_pm7(z, xyz)
    o = harness.run(z, xyz)
    assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-5


def _footprint_bytes(mol):
    with api.Engine() as eng:
        done, r = eng.poll(eng.submit(*mol, want_matrices=0), wait=True)
        assert done and not isinstance(r, Exception)
        return eng.stats()["peak_bytes"]


def test_hbm_budget_queues_requests_and_results_do_not_change():
    mols = [G.water_cluster(30, seed=s) for s in range(6)]
    alone = []
    for m in mols:
        with api.Engine() as eng:
            done, r = eng.poll(eng.submit(*m, want_matrices=0), wait=True)
            assert done and not isinstance(r, Exception)
            alone.append(r)
    fp = _footprint_bytes(mols[0])
    budget_mb = int(math.ceil(2.5 * fp / 2 ** 20))
    with api.Engine(hbm_budget_mb=budget_mb) as eng:
        tickets = [eng.submit(*m, want_matrices=0) for m in mols]
        res = [eng.poll(t, wait=True)[1] for t in tickets]
        st = eng.stats()
    assert st["budget_bytes"] == budget_mb * 2 ** 20
    assert st["admitted"] == len(mols)
    assert 1 <= st["peak_active"] <= 3 < len(mols), st  # the rest waited for memory
    assert st["peak_bytes"] <= st["budget_bytes"], st
    for a, b in zip(alone, res):
        assert not isinstance(b, Exception)
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1e-9
        assert np.max(np.abs(a["charges"] - b["charges"])) < 1e-10
    # later requests waited for earlier ones to leave
    lat = [r["latency_ms"] for r in res]
    assert max(lat) > min(lat)


def test_budget_below_one_footprint_still_serves_one_at_a_time():
    mols = [G.water_cluster(12, seed=s) for s in range(3)]
    with api.Engine(hbm_budget_mb=1) as eng:
        res = [eng.poll(t, wait=True)[1] for t in [eng.submit(*m, want_matrices=0) for m in mols]]
        st = eng.stats()
    assert st["peak_active"] == 1 and st["admitted"] == 3
    for m, r in zip(mols, res):
        o = harness.run(*m, want_matrices=0)
        assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1e-5


def test_run_sharded_on_one_rank_uses_the_batched_engine():
    mols = [G.water_cluster(k, seed=k) for k in (2, 7, 15)] + [G.alkane(n, seed=n) for n in (4, 11)]
    mols.append((np.array([1, 1], np.uint8), np.zeros((2, 3))))  # coincident atoms: an error result
    before = api.launch_count()
    res = shard.run_sharded(mols, want_matrices=0)
    assert api.launch_count() > before
    direct = api.run_batch(mols, want_matrices=0)
    for r, d, m in zip(res, direct, mols):
        if isinstance(d, api.Pm7Error):
            assert isinstance(r, api.Pm7Error) and r.code == d.code
            continue
        assert r["heat_of_formation_kcal"] == d["heat_of_formation_kcal"]
        s = api.run_pm7(*m, want_matrices=0)
        assert abs(r["heat_of_formation_kcal"] - s["heat_of_formation_kcal"]) < 1e-7
