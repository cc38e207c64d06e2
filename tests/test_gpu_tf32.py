"""The tcgen05 (kind::tf32) squaring of the mixed-precision SP2 against fp64.

X is split as tf32(X) + remainder and X X accumulated in fp32 in tensor memory (3xTF32),
so the product carries about fp32 accuracy; the tensor core's fp32 accumulation is not
round-to-nearest, so the error grows with the inner dimension: 4e-8 n of the largest
element is allowed. Checked on symmetric matrices shaped like SP2 iterates (spectrum in
[0, 1]) at sizes that cover one tile, ragged tiles and several tile rows.
"""
import numpy as np
import pytest

from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu


def _iterate(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    lam = rng.uniform(0.0, 1.0, size=n)
    return (q * lam) @ q.T


@pytest.mark.parametrize("n", [40, 128, 131, 300, 517])
def test_square_matches_fp64(n):
    x = _iterate(n, n)
    c = api.square_tf32(x)
    ref = x @ x
    err = np.max(np.abs(c - ref)) / np.max(np.abs(ref))
    assert err < 4e-8 * max(n, 64), err
    assert np.array_equal(c, c.T)  # written once and mirrored


@pytest.mark.parametrize("n", [40, 128, 131, 300, 517])
def test_product_matches_fp64(n):
    # the DIIS commutator product F P of the fp32 cycles: two different symmetric operands,
    # a Fock-like one with a wide spectrum and an SP2-like one in [0, 1]
    rng = np.random.default_rng(n + 1)
    f = rng.normal(size=(n, n))
    f = 0.5 * (f + f.T) * 10.0 + np.diag(np.linspace(-40.0, 20.0, n))
    p = _iterate(n, n + 2)
    c = api.product_tf32(f, p)
    ref = f @ p
    err = np.max(np.abs(c - ref)) / np.max(np.abs(ref))
    assert err < 4e-8 * max(n, 64), err
    assert not np.array_equal(c, c.T)  # every tile written, no mirror


def test_square_is_deterministic():
    x = _iterate(300, 3)
    assert np.array_equal(api.square_tf32(x), api.square_tf32(x))


def test_mixed_precision_scf_matches_fp64_oracle():
    # fp32 (tcgen05) densities for the early cycles, fp64 refinement cycles at the end:
    # the heat of formation within 1e-4 kcal/mol and the charges within 1e-5 e of the oracle
    # (another trajectory stops elsewhere inside the same p_tol window)
    from oracle import harness
    from pm7b200 import geometry as G

    z, x = G.water_cluster(100, seed=2)  # 600 basis functions: the SP2 path
    r = api.run_pm7(z, x, precision=1)
    o = harness.run(z, x)
    assert r["fp32_iterations"] > 0
    assert r["iterations"] > r["fp32_iterations"]
    assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1.0e-4
    assert np.max(np.abs(r["charges"] - o["charges"])) < 1.0e-5
    f = api.run_pm7(z, x)
    assert f["fp32_iterations"] == 0


@pytest.mark.parametrize("case", ["water30", "chain_s_cl"])
def test_fp32_fock_build_against_fp64(case):
    # the Fock build of the mixed-precision mode's early cycles (density and stored pair
    # integrals read as float, sums in FP32) against the FP64 build, which matches the oracle
    # to 1e-10 eV: a converged RHF density of a water cluster and of a chain with S and Cl
    # (the MNDO/d one-centre block)
    if case == "water30":
        z, x = G.water_cluster(30, seed=4)
    else:
        z, x = G.substituted_chain(14, np.random.default_rng(5), p_s=0.3, p_cl=0.3)
    r = api.run_pm7(z, x, want_matrices=1)
    p = np.asarray(r["density"])
    f64 = api.fock(z, x, p, 0.5 * p)
    f32 = api.fock(z, x, p, 0.5 * p, fp32=True)
    scale = np.max(np.abs(f64))
    err = np.max(np.abs(f32 - f64))
    assert err < 2e-6 * scale, (err, scale)
    assert err > 0.0  # the FP32 kernels ran, not the FP64 ones
