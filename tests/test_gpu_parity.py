"""Device parity: every stage and the whole `run_pm7` against the CPU oracle.

The oracle is pinned to the reference's recorded results (test_oracle_golden.py); here
the device path must match it on the same inputs: 1e-10 (absolute, eV) for integrals,
H_core and Fock elements, and for converged runs 1e-5 kcal/mol in the heat of formation,
1e-7 eV per atom in the total energy and 1e-6 e in the Mulliken charges.
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


def _sp_cases(golden):
    out = []
    for name, case in sorted(golden.items()):
        els = {line.split()[0] for line in case["atoms"]}
        if els <= SP_ONLY:
            out.append(name)
    return out


@pytest.mark.parametrize("zi,zj", [(1, 1), (6, 1), (8, 1), (6, 6), (8, 8), (7, 8), (9, 6), (5, 1), (12, 8)])
@pytest.mark.parametrize("r_ang", [0.95, 1.5, 2.7, 6.9, 7.4])
def test_pair_blocks(zi, zj, r_ang):
    rng = np.random.default_rng(zi * 100 + zj)
    v = rng.normal(size=3)
    d = v / np.linalg.norm(v) * r_ang / harness.A0
    w, e1b, e2a, s = api.pair(zi, zj, d)
    wo, e1o, e2o, so = harness.pair(zi, zj, d)
    assert w.shape == wo.shape
    np.testing.assert_allclose(w, wo, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(e1b, e1o, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(e2a, e2o, rtol=0, atol=INT_TOL)
    np.testing.assert_allclose(s, so, rtol=0, atol=INT_TOL)


def test_pair_axis_aligned():
    # the exact rotation-frame antipode (bond along -x after the frame flip)
    for d in ([1.3, 0.0, 0.0], [-1.3, 0.0, 0.0], [0.0, 0.0, 2.1]):
        w, e1b, e2a, s = api.pair(8, 6, np.array(d) / harness.A0)
        wo, e1o, e2o, so = harness.pair(8, 6, np.array(d) / harness.A0)
        np.testing.assert_allclose(w, wo, rtol=0, atol=INT_TOL)
        np.testing.assert_allclose(s, so, rtol=0, atol=INT_TOL)


def _cluster(k, seed):
    return G.water_cluster(k, seed=seed)


def test_core_hamiltonian_water_cluster():
    z, x = _cluster(40, 5)  # spans more than 7 Angstrom: near and far pairs
    h = api.core_hamiltonian(z, x)
    ho = harness.core_hamiltonian(z, x)
    assert np.max(np.abs(h - ho)) < INT_TOL * 10


def test_core_hamiltonian_alkane():
    z, x = G.alkane(12, seed=2)
    np.testing.assert_allclose(api.core_hamiltonian(z, x), harness.core_hamiltonian(z, x), rtol=0, atol=INT_TOL)


def _random_density(nao, rng):
    a = rng.normal(size=(nao, nao)) * 0.1
    p = a @ a.T / nao
    np.fill_diagonal(p, np.abs(np.diag(p)) + 0.5)
    return p


def test_fock_rhf_and_spin():
    rng = np.random.default_rng(11)
    z, x = _cluster(30, 7)
    nao = int(sum(1 if zz == 1 else 4 for zz in z))
    pt = _random_density(nao, rng)
    ps = 0.5 * pt
    f = api.fock(z, x, pt, ps)
    fo = harness.fock(z, x, pt, ps)
    assert np.max(np.abs(f - fo)) < INT_TOL * 10
    pa = _random_density(nao, rng)
    f2 = api.fock(z, x, pt, pa)
    fo2 = harness.fock(z, x, pt, pa)
    assert np.max(np.abs(f2 - fo2)) < INT_TOL * 10


def test_core_core_and_corrections():
    for z, x in (_cluster(27, 3), G.alkane(8, seed=1), G.decane(4)):
        assert abs(api.core_core(z, x) - harness.core_core(z, x)) < 1e-9 * max(1.0, abs(harness.core_core(z, x)))
        c = api.corrections(z, x)
        co = harness.corrections(z, x)
        np.testing.assert_allclose(c, co, rtol=1e-11, atol=1e-11)
    z, x = _cluster(8, 9)
    np.testing.assert_allclose(api.corrections(z, x, smooth=True), harness.corrections(z, x, smooth=True),
                               rtol=1e-11, atol=1e-11)


def _compare_runs(name, r, o, n_atoms):
    assert r["iterations"] >= 1
    assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL, name
    assert abs(r["total_ev"] - o["total_ev"]) < E_TOL_PER_ATOM * n_atoms, name
    assert np.max(np.abs(r["charges"] - o["charges"])) < Q_TOL, name
    np.testing.assert_allclose(r["dipole_debye"], o["dipole_debye"], rtol=0, atol=1e-5)


def test_run_golden_sp_cases(golden):
    names = _sp_cases(golden)
    assert len(names) > 60
    bad = []
    for name in names:
        case = golden[name]
        z, x = harness.parse_lines(case["atoms"])
        kw = dict(charge=float(case["charge"]), multiplicity=case["multiplicity"])
        try:
            o = harness.run(z, x, **kw)
        except harness.OracleError as e:
            if e.code == 4:
                continue
            raise
        try:
            r = api.run_pm7(z, x, **kw)
        except api.Pm7Error as e:
            if e.code == 4:
                continue
            bad.append(f"{name}: {e}")
            continue
        ref = case["pm7_rs"]
        if abs(r["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) > DHF_TOL:
            bad.append(f"{name}: dHf {r['heat_of_formation_kcal']} vs reference {ref['heat_of_formation_kcal']}")
        try:
            _compare_runs(name, r, o, len(z))
        except AssertionError as e:
            bad.append(f"{name}: {e}")
    assert not bad, "\n".join(bad)


def test_run_decane_and_clusters():
    for z, x in (G.decane(0), G.decane(7), _cluster(27, 2), G.alkane(20, seed=5)):
        o = harness.run(z, x)
        r = api.run_pm7(z, x)
        _compare_runs("generated", r, o, len(z))
        assert r["device_ms"] > 0


def test_uhf_radicals(golden):
    for name in ("methyl_radical", "hydroxyl_radical", "oxygen_triplet", "allyl_radical", "nitric_oxide"):
        case = golden[name]
        z, x = harness.parse_lines(case["atoms"])
        kw = dict(charge=float(case["charge"]), multiplicity=case["multiplicity"])
        r = api.run_pm7(z, x, **kw)
        assert r["unrestricted"] == 1
        o = harness.run(z, x, **kw)
        _compare_runs(name, r, o, len(z))


def test_forced_uhf_closed_shell_and_options():
    z, x = G.decane(3)
    o = harness.run(z, x, reference="uhf")
    r = api.run_pm7(z, x, reference="uhf")
    _compare_runs("uhf-closed", r, o, len(z))
    for kw in (dict(accelerator="cdiis"), dict(accelerator="none", max_scf=400), dict(level_shift=2.0)):
        o = harness.run(z, x, **kw)
        r = api.run_pm7(z, x, **kw)
        _compare_runs(str(kw), r, o, len(z))


def test_errors_mirror_the_reference():
    z, x = G.decane(0)
    with pytest.raises(api.Pm7Error) as info:
        api.run_pm7(z, x, max_scf=1)
    assert info.value.code == 6  # ScfNotConverged: an error with no result
    with pytest.raises(api.Pm7Error) as info:
        api.run_pm7(z, x, max_memory_mb=1)
    assert info.value.code == 8
    with pytest.raises(api.Pm7Error) as info:
        api.run_pm7(np.array([118], dtype=np.uint8), np.zeros((1, 3)))
    assert info.value.code == 2


def test_initial_density_warm_start():
    z, x = G.decane(1)
    r0 = api.run_pm7(z, x)
    r1 = api.run_pm7(z, x, initial_density=r0["density"])
    assert r1["iterations"] <= 3
    assert abs(r1["heat_of_formation_kcal"] - r0["heat_of_formation_kcal"]) < DHF_TOL


def test_matrices_are_consistent():
    z, x = G.decane(2)
    r = api.run_pm7(z, x)
    c = r["mo_coeff"]
    nocc = r["n_occ"]
    p = 2.0 * c[:, :nocc] @ c[:, :nocc].T
    assert np.max(np.abs(p - r["density"])) < 1e-8
    assert np.allclose(c.T @ c, np.eye(c.shape[0]), atol=1e-10)
    assert np.all(np.diff(r["mo_energies"]) >= -1e-12)


def test_deterministic_bits():
    z, x = _cluster(20, 4)
    a = api.run_pm7(z, x)
    b = api.run_pm7(z, x)
    assert a["heat_of_formation_kcal"] == b["heat_of_formation_kcal"]
    assert np.array_equal(a["density"], b["density"])


def _with_solver(name, fn):
    import os

    old = os.environ.get("PM7_DENSITY_SOLVER")
    os.environ["PM7_DENSITY_SOLVER"] = name
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["PM7_DENSITY_SOLVER"]
        else:
            os.environ["PM7_DENSITY_SOLVER"] = old


def test_sp2_purification_matches_diagonalisation():
    # SP2 builds the same aufbau projector as the eigendecomposition, so the SCF takes the
    # same path and lands on the same converged state.
    for z, x in (_cluster(90, 8), G.decane(5)):
        a = _with_solver("sp2", lambda: api.run_pm7(z, x))
        b = _with_solver("syevd", lambda: api.run_pm7(z, x))
        o = harness.run(z, x)
        assert a["iterations"] == b["iterations"]
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1e-7
        assert np.max(np.abs(a["density"] - b["density"])) < 1e-8
        np.testing.assert_allclose(a["mo_energies"], b["mo_energies"], rtol=0, atol=1e-8)
        _compare_runs("sp2", a, o, len(z))


def test_sp2_uhf():
    z, x = _cluster(30, 1)
    a = _with_solver("sp2", lambda: api.run_pm7(z, x, reference="uhf"))
    o = harness.run(z, x, reference="uhf")
    _compare_runs("sp2-uhf", a, o, len(z))


def test_jacobi_eigensolver_matches_the_library_one():
    # the Jacobi kernel (orders <= 112, warm-started from the previous iteration's vectors)
    # and cuSOLVER's dsyevd take the same SCF path to the same state, RHF and UHF
    for z, x, kw in ((*G.decane(3), {}), (*_cluster(15, 4), {}), (*_cluster(10, 2), {"reference": "uhf"})):
        a = _with_solver("jacobi", lambda: api.run_pm7(z, x, **kw))
        b = _with_solver("syevd", lambda: api.run_pm7(z, x, **kw))
        o = harness.run(z, x, **kw)
        assert a["iterations"] == b["iterations"]
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1e-7
        assert np.max(np.abs(a["density"] - b["density"])) < 1e-8
        np.testing.assert_allclose(a["mo_energies"], b["mo_energies"], rtol=0, atol=1e-8)
        _compare_runs("jacobi", a, o, len(z))
