"""The engine's divide-and-conquer partition (host code, no device) against the oracle's
restatement of src/dandc/partition.rs, and the properties the reference's partition tests
assert: every atom is the core of exactly one subsystem, and the subsystem size stays flat as a
chain grows."""
import numpy as np
import pytest

from oracle import harness
from pm7b200 import api
from pm7b200 import geometry as G


def chain(n, spacing=2.0):
    z = np.ones(n, dtype=np.uint8)
    x = np.zeros((n, 3))
    x[:, 0] = spacing * np.arange(n)
    return z, x


CASES = [
    ("alkane10", lambda: G.flat_alkane(10), 6, 6.0),
    ("alkane10_wide", lambda: G.flat_alkane(10), 6, 30.0),
    ("alkane40", lambda: G.flat_alkane(40), 8, 15.0),
    ("alkane160", lambda: G.flat_alkane(160), 8, 15.0),
    ("hchain", lambda: chain(40), 5, 6.0),
    ("water100", lambda: G.water_cluster(100, seed=3), 12, 10.0),
    ("water100_core1", lambda: G.water_cluster(100, seed=3), 1, 5.0),
    ("sclchain", lambda: G.substituted_chain(30, np.random.default_rng(2), p_s=0.3, p_cl=0.2), 7, 9.0),
]


@pytest.mark.parametrize("name, make, core, buffer", CASES, ids=[c[0] for c in CASES])
def test_partition_matches_the_oracle(name, make, core, buffer):
    z, x = make()
    d = api.dandc_partition(z, x, core_size=core, buffer=buffer)
    o = harness.dandc_partition(z, x, core_size=core, buffer=buffer)
    assert np.array_equal(d[0], o[0])
    assert np.array_equal(d[1], o[1])
    assert d[2] == o[2]


def test_every_atom_is_the_core_of_exactly_one_subsystem():
    z, x = chain(40)
    core_of, sizes, _ = api.dandc_partition(z, x, core_size=5, buffer=6.0)
    counts = np.bincount(core_of, minlength=len(sizes))
    assert counts.sum() == 40 and (counts >= 1).all() and (counts <= 5).all()


def test_subsystem_size_stays_flat_as_the_system_grows():
    # partition.rs subsystem_size_stays_flat_as_the_system_grows
    _, small, _ = api.dandc_partition(*chain(40), core_size=5, buffer=6.0)
    _, large, _ = api.dandc_partition(*chain(160), core_size=5, buffer=6.0)
    assert len(large) == 4 * len(small)
    assert large.max() <= small.max() + 1


def test_invalid_arguments_are_refused():
    z, x = chain(4)
    with pytest.raises(api.Pm7Error):
        api.dandc_partition(z, x, core_size=0)
    with pytest.raises(api.Pm7Error):
        api.dandc_partition(z, x, buffer=0.0)
