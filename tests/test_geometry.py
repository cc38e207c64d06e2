"""Workload generators: seeded, chemically sane, and of the documented sizes (CPU)."""
import numpy as np

from pm7b200 import geometry as G

A0 = 0.529177210903


def _dists(x):
    d = np.linalg.norm(x[:, None] - x[None], axis=-1)
    np.fill_diagonal(d, np.inf)
    return d


def test_decane_shape_and_seed():
    z, x = G.decane(0)
    assert len(z) == 32 and (z == 6).sum() == 10
    z2, x2 = G.decane(0)
    assert np.array_equal(x, x2)
    assert not np.array_equal(x, G.decane(1)[1])
    d = _dists(x * A0)
    assert d.min() > 1.0


def test_water_cluster_sizes():
    for k, atoms in ((334, 1002), (1000, 3000)):
        z, x = G.water_cluster(k, seed=0)
        assert len(z) == atoms
        d = _dists(x[:300] * A0)
        assert d.min() > 0.9


def test_batch_mixture():
    mols = G.batch(16, seed=3)
    assert len(mols) == 16
    sizes = [len(z) for z, _ in mols]
    assert min(sizes) >= 5 and max(sizes) <= 192
