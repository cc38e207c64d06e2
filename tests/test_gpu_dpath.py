"""Device parity in the MNDO/d frame and for heavy sp shells, against the CPU oracle.

A molecule with any d-shell atom (S, Cl, P, Si, Al, Br, I, the transition metals, ...)
is evaluated entirely in the MNDO/d frame (pm7-rs src/hamiltonian.rs:346-355): the
multipole integrals of src/mndod_twocenter.rs and the general Slater overlaps of
src/overlap_d.rs for every pair. sp elements with valence n >= 4 (K, Ca, Zn, Ge, Se, Sn,
...) take the numerical overlaps of src/overlap_numeric.rs. Tolerances as in
test_gpu_parity.py: 1e-10 eV for integrals and matrix elements, 1e-5 kcal/mol in the
heat of formation, 1e-7 eV per atom in the total energy, 1e-6 e in the charges.
"""
import numpy as np
import pytest

from oracle import harness
from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu

INT_TOL = 1.0e-10
DHF_TOL = 1.0e-5
Q_TOL = 1.0e-6
E_TOL_PER_ATOM = 1.0e-7

SP_ONLY = set("H He Li Be B C N O F Ne Na Mg".split())

# (heavier, lighter): d-d, d-sp, d-H, transition metals with iod > 0 (PM7 d balance)
D_PAIRS = [(16, 1), (17, 6), (17, 17), (15, 8), (14, 1), (13, 17), (35, 35), (53, 6),
           (26, 6), (26, 1), (22, 17), (29, 29), (44, 7), (74, 9), (78, 17), (79, 1)]
# sp elements whose valence shell has n >= 4: numerical overlaps
HEAVY_SP_PAIRS = [(30, 1), (32, 6), (34, 8), (50, 1), (38, 8), (19, 9), (30, 30), (52, 1)]


def _direction(seed):
    v = np.random.default_rng(seed).normal(size=3)
    return v / np.linalg.norm(v)


def _check_pair(zi, zj, d, force_dpath=False):
    w, e1b, e2a, s = api.pair(zi, zj, d, force_dpath=force_dpath)
    wo, e1o, e2o, so = harness.pair(zi, zj, d, force_dpath=force_dpath)
    assert w.shape == wo.shape
    np.testing.assert_allclose(w, wo, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(e1b, e1o, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(e2a, e2o, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(s, so, rtol=0, atol=INT_TOL)


@pytest.mark.parametrize("zi,zj", D_PAIRS)
@pytest.mark.parametrize("r_ang", [0.9, 1.6, 2.8, 6.9, 7.5])
def test_pair_blocks_d(zi, zj, r_ang):
    _check_pair(zi, zj, _direction(zi * 131 + zj) * r_ang / harness.A0)


@pytest.mark.parametrize("zi,zj", [(1, 1), (6, 1), (8, 8), (7, 6), (9, 1)])
def test_pair_blocks_forced_dframe(zi, zj):
    for r_ang in (1.1, 3.3, 7.2):
        _check_pair(zi, zj, _direction(zi + 7 * zj) * r_ang / harness.A0, force_dpath=True)


def test_pair_blocks_d_axis_aligned():
    # the rotation's polar axis, where the azimuth is undefined (rotmat's sb < 1e-7 branch)
    for d in ([0.0, 0.0, 2.4], [0.0, 0.0, -2.4], [2.4, 0.0, 0.0], [0.0, -2.4, 0.0]):
        _check_pair(17, 6, np.array(d) / harness.A0)
        _check_pair(26, 17, np.array(d) / harness.A0)


@pytest.mark.parametrize("zi,zj", HEAVY_SP_PAIRS)
@pytest.mark.parametrize("r_ang", [1.2, 2.5, 5.0])
def test_pair_blocks_heavy_sp(zi, zj, r_ang):
    _check_pair(zi, zj, _direction(zi * 17 + zj) * r_ang / harness.A0)


def _sulfur_cluster(k, seed, n_sub):
    """A water cluster with n_sub oxygens turned into sulfur (an input, not a chemistry claim)."""
    z, x = G.water_cluster(k, seed=seed)
    z = np.array(z, dtype=np.int32)
    oxy = np.flatnonzero(z == 8)
    z[oxy[:n_sub]] = 16
    return z, x


def test_core_hamiltonian_d_cluster():
    z, x = _sulfur_cluster(40, 5, 3)  # spans more than 7 Angstrom: near and far pairs in the d frame
    h = api.core_hamiltonian(z, x)
    ho = harness.core_hamiltonian(z, x)
    assert h.shape == ho.shape
    assert np.max(np.abs(h - ho)) < INT_TOL * 10


def test_core_hamiltonian_forced_dframe():
    z, x = G.alkane(6, seed=4)
    h = api.core_hamiltonian(z, x, force_dpath=True)
    ho = harness.core_hamiltonian(z, x, force_dpath=True)
    np.testing.assert_allclose(h, ho, rtol=0, atol=INT_TOL)
    # the two frames are two evaluations of one model: close, but not equal to rounding
    np.testing.assert_allclose(h, api.core_hamiltonian(z, x), rtol=0, atol=1e-5)


def test_fock_d_cluster():
    rng = np.random.default_rng(3)
    z, x = _sulfur_cluster(30, 7, 4)
    nao = int(sum(1 if zz == 1 else (9 if zz == 16 else 4) for zz in z))
    a = rng.normal(size=(nao, nao)) * 0.1
    pt = a @ a.T / nao
    np.fill_diagonal(pt, np.abs(np.diag(pt)) + 0.5)
    f = api.fock(z, x, pt, 0.5 * pt)
    fo = harness.fock(z, x, pt, 0.5 * pt)
    assert np.max(np.abs(f - fo)) < INT_TOL * 10


def _compare_runs(name, r, o, n_atoms):
    assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL, name
    assert abs(r["total_ev"] - o["total_ev"]) < E_TOL_PER_ATOM * n_atoms, name
    assert np.max(np.abs(r["charges"] - o["charges"])) < Q_TOL, name
    np.testing.assert_allclose(r["dipole_debye"], o["dipole_debye"], rtol=0, atol=1e-5)


def test_run_golden_d_and_heavy_cases(golden):
    names = [n for n, c in sorted(golden.items()) if not {l.split()[0] for l in c["atoms"]} <= SP_ONLY]
    assert len(names) >= 95
    bad = []
    for name in names:
        case = golden[name]
        z, x = harness.parse_lines(case["atoms"])
        kw = dict(charge=float(case["charge"]), multiplicity=case["multiplicity"])
        try:
            r = api.run_pm7(z, x, **kw)
        except api.Pm7Error as e:
            bad.append(f"{name}: {e}")
            continue
        ref = case["pm7_rs"]
        if abs(r["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) > DHF_TOL:
            bad.append(f"{name}: dHf {r['heat_of_formation_kcal']} vs reference {ref['heat_of_formation_kcal']}")
            continue
        try:
            _compare_runs(name, r, harness.run(z, x, **kw), len(z))
        except AssertionError as e:
            bad.append(f"{name}: {e}")
    assert not bad, "\n".join(bad)


def test_run_d_cluster_and_forced_frame():
    z, x = _sulfur_cluster(24, 11, 2)
    _compare_runs("sulfur cluster", api.run_pm7(z, x), harness.run(z, x), len(z))
    z, x = G.decane(3)
    r = api.run_pm7(z, x, force_dpath=True)
    _compare_runs("decane, d frame", r, harness.run(z, x, force_dpath=True), len(z))
    # the frames differ at the 1e-4 kcal/mol level (their multipole charge separations differ)
    assert abs(r["heat_of_formation_kcal"] - api.run_pm7(z, x)["heat_of_formation_kcal"]) < 1e-2
