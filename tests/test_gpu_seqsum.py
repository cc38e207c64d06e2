"""The reference-order sum on the device (pm7_stage_seqsum) against a serial loop.

pm7-rs adds its energies with plain left-to-right folds (`Matrix::frobenius_dot`,
src/linalg.rs:138-141; `core_core_energy`, src/repulsion.rs:16-36). The engine reproduces
those folds exactly, in parallel; these tests require the same bits as a serial loop on
inputs built to reach every path of the kernel: running sums that cross binades, exact
ties on the rounding grid, cancellation, zeros, non-finite terms and chunk edges.
"""
import math

import numpy as np
import pytest

from oracle import harness
from pm7b200 import api
from pm7b200 import geometry as G


def fold(a, b=None):
    """Serial left-to-right sum (numpy's accumulate adds one element at a time)."""
    t = np.asarray(a, np.float64) if b is None else np.asarray(a, np.float64) * np.asarray(b, np.float64)
    t = t.reshape(-1)
    with np.errstate(over="ignore", invalid="ignore"):
        return -0.0 if t.size == 0 else float(np.add.accumulate(t)[-1])


def bits(x):
    return int(np.float64(x).view(np.int64))


def same(x, y):
    return (math.isnan(x) and math.isnan(y)) or bits(x) == bits(y)


def cases():
    rng = np.random.default_rng(7)
    c = {
        "normal": (rng.standard_normal(100_000), None),
        "mixed_magnitudes": (rng.choice([-1.0, 1.0], 60_000) * 10.0 ** rng.uniform(-20, 6, 60_000), None),
        "growing": (np.abs(rng.standard_normal(50_000)) * np.linspace(1, 1e4, 50_000), None),
        "cancellation": (np.repeat([1e6, -1e6 + 1e-3], 20_000) + rng.standard_normal(40_000) * 1e-6, None),
        "grid_ties": (np.concatenate([[2.0 ** 53], np.ones(9000), rng.integers(-3, 4, 9000).astype(float)]), None),
        "half_ties": (np.concatenate([[2.0 ** 52], np.full(9000, 0.5), np.full(9000, 1.5)]), None),
        "zeros": (np.zeros(10_000), None),
        "negative_zeros": (-np.zeros(5000), None),
        "two": (np.array([3.0, -1.0]), None),
        "one": (np.array([-2.5]), None),
        "empty": (np.zeros(0), None),
        "chunk_minus_one": (rng.standard_normal(4095) + 100.0, None),
        "chunk": (rng.standard_normal(4096) + 100.0, None),
        "chunk_plus_one": (rng.standard_normal(4097) + 100.0, None),
        "two_chunks_plus_one": (rng.standard_normal(8193) - 50.0, None),
        "subnormal": (rng.standard_normal(10_000) * 1e-310, None),
        "nan_inside": (np.concatenate([rng.standard_normal(5000), [np.nan], rng.standard_normal(5000)]), None),
        "inf_inside": (np.concatenate([rng.standard_normal(5000) + 1.0, [np.inf], rng.standard_normal(5000)]), None),
        "overflow": (np.array([1e308, 1e308, -1e308, 5.0]), None),
        "products": (rng.standard_normal(1_000_003), rng.standard_normal(1_000_003)),
    }
    # the shape of <P, H> at the engine's sizes: a large negative diagonal term every
    # nao + 1 elements, small off-diagonal products in between
    nao = 2004
    t = rng.standard_normal(nao * nao) * 1e-3
    t[:: nao + 1] = -1.0e3 * rng.uniform(1, 4, nao)
    c["energy_like"] = (t, None)
    c["energy_like_products"] = (t, 1.0 + 1e-9 * rng.standard_normal(t.size))
    return c


CASES = cases()


def test_fold_is_a_serial_loop():
    # the test's own yardstick: accumulate equals an explicit Python loop
    rng = np.random.default_rng(3)
    a = rng.standard_normal(20_000) * 10.0 ** rng.uniform(-8, 8, 20_000)
    s = -0.0
    for v in a.tolist():
        s = s + v
    assert bits(fold(a)) == bits(s)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_seqsum_matches_the_serial_fold_bit_for_bit(name):
    a, b = CASES[name]
    got = api.seqsum(a, b)
    want = fold(a, b)
    assert same(got, want), (name, got, want)


@pytest.mark.gpu
def test_seqsum_of_a_density_and_core_hamiltonian():
    z, x = G.water_cluster(60, seed=2)
    h = api.core_hamiltonian(z, x)
    rng = np.random.default_rng(11)
    p = rng.standard_normal(h.shape) * 1e-2
    p = p + p.T + np.diag(rng.uniform(0.5, 1.5, h.shape[0]))
    assert same(api.seqsum(p, h), fold(p, h))


@pytest.mark.gpu
def test_core_core_is_the_reference_fold():
    # per-pair energies agree to an ulp or two; summed in pair order like the reference,
    # the totals agree to a few ulps of the sum (an accurate sum would differ by ~3e-7 eV)
    z, x = G.water_cluster(334, seed=0)
    dev = api.core_core(z, x)
    ora = harness.core_core(z, x)
    assert abs(dev - ora) <= 8 * np.spacing(abs(ora)), (dev, ora, (dev - ora) / np.spacing(abs(ora)))
