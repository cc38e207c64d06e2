"""Eigenvalues without eigenvectors on the device (cluster tridiagonalisation + Sturm).

The reported MO energies (pm7-rs src/scf.rs:1299-1305 via src/linalg.rs:231-278) come
from this path whenever no orbitals are returned. Checked against LAPACK (numpy) on
random and structured symmetric matrices, and inside run_pm7 / run_batch against the
full eigendecomposition the same engine does when orbitals are returned.
"""
import numpy as np
import pytest

from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu


def _sym(n, seed, scale=10.0):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) * scale
    return 0.5 * (a + a.T)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 32, 33, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 700, 1024, 1100])
def test_random_symmetric_matches_lapack(n):
    a = _sym(n, n)
    (w,) = api.eigenvalues([a])
    ref = np.linalg.eigvalsh(a)
    tol = 1e-12 * max(1.0, np.abs(ref).max()) * max(1.0, np.sqrt(n))
    assert np.max(np.abs(w - ref)) < tol


def test_fock_sized_matrix_matches_lapack():
    n = 2004
    a = _sym(n, 7, scale=3.0) + np.diag(np.linspace(-40.0, 60.0, n))
    (w,) = api.eigenvalues([a])
    ref = np.linalg.eigvalsh(a)
    assert np.max(np.abs(w - ref)) < 1e-9


def test_structured_matrices():
    n = 150
    mats = [np.diag(np.arange(n, 0, -1.0)),                       # already diagonal: no reflection
            np.eye(n) * 3.0 + 1e-9 * _sym(n, 1),                   # clustered spectrum
            np.ones((n, n)),                                       # rank one
            np.zeros((40, 40)),                                    # all zero
            np.diag(np.ones(n - 1), 1) + np.diag(np.ones(n - 1), -1)]  # tridiagonal already
    ws = api.eigenvalues(mats)
    for m, w in zip(mats, ws):
        ref = np.linalg.eigvalsh(m)
        assert np.max(np.abs(w - ref)) < 1e-11 * max(1.0, np.abs(ref).max()), m.shape


def test_many_orders_in_one_call_equal_one_by_one_and_are_deterministic():
    orders = [3, 140, 600, 40, 1030, 260, 9]  # several cluster sizes in one call
    mats = [_sym(n, 100 + n) for n in orders]
    together = api.eigenvalues(mats)
    again = api.eigenvalues(mats)
    for m, w, w2 in zip(mats, together, again):
        (alone,) = api.eigenvalues([m])
        assert np.array_equal(w, alone)
        assert np.array_equal(w, w2)


def test_run_pm7_energies_without_matrices_match_full_eigensolve():
    for z, x in (G.water_cluster(40, seed=3), G.alkane(12, seed=1)):
        full = api.run_pm7(z, x, want_matrices=1)
        lean = api.run_pm7(z, x, want_matrices=0)
        assert lean["iterations"] == full["iterations"]
        np.testing.assert_allclose(lean["mo_energies"], full["mo_energies"], rtol=0, atol=1e-9)
        assert abs(lean["homo_ev"] - full["homo_ev"]) < 1e-9 and abs(lean["lumo_ev"] - full["lumo_ev"]) < 1e-9


def test_batch_energies_without_matrices_match_full_eigensolve():
    mols = [G.water_cluster(k, seed=k) for k in (2, 30, 70)] + [G.alkane(n, seed=n) for n in (1, 9, 33)]
    full = api.run_batch(mols, want_matrices=1)
    lean = api.run_batch(mols, want_matrices=0)
    for a, b in zip(full, lean):
        np.testing.assert_allclose(b["mo_energies"], a["mo_energies"], rtol=0, atol=1e-9)
        assert abs(b["heat_of_formation_kcal"] - a["heat_of_formation_kcal"]) < 1e-10
