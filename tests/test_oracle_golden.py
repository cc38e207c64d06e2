"""The CPU oracle against the reference's own recorded results.

Every case geometry is regenerated by pm7-rs tools/oracle/baseline.py and every
expected value is pm7-rs's own `run_pm7` output recorded in
tools/oracle/baselines/reference.json (see tests/golden/make_golden.py). The oracle
must reproduce them to 1e-6 kcal/mol in the heat of formation, 1e-6 e in the Mulliken
charges and 1e-7 eV per atom in the total energy before any device result is compared
with it.
"""
import numpy as np
import pytest

from oracle import harness

DHF_TOL = 1.0e-6      # kcal/mol
Q_TOL = 1.0e-6        # e
E_TOL_PER_ATOM = 1.0e-7  # eV
ORB_TOL = 1.0e-5      # eV (HOMO/LUMO; degenerate frontier levels are ordering-sensitive)


def _cases(golden):
    return sorted(golden)


def test_golden_cases(golden):
    checked, failures = 0, []
    for name in _cases(golden):
        case = golden[name]
        z, xyz = harness.parse_lines(case["atoms"])
        r = harness.run(z, xyz, charge=float(case["charge"]), multiplicity=case["multiplicity"])
        ref = case["pm7_rs"]
        n = len(z)
        checks = [
            ("dHf", r["heat_of_formation_kcal"], ref["heat_of_formation_kcal"], DHF_TOL),
            ("energy", r["total_ev"], ref["energy_ev"], E_TOL_PER_ATOM * n),
        ]
        dq = float(np.max(np.abs(r["charges"] - np.array(ref["charges"])))) if n else 0.0
        if dq > Q_TOL:
            failures.append(f"{name}: charges off by {dq:.2e}")
        for label, got, want, tol in checks:
            if abs(got - want) > tol:
                failures.append(f"{name}: {label} {got!r} vs {want!r}")
        checked += 1
    assert not failures, "\n".join(failures)
    # Every recorded case, sp and MNDO/d elements alike (s, p, d shells; H..No).
    assert checked == len(golden) >= 175, checked


def test_water_known_answer():
    # pm7-rs src/scf.rs:2153-2168: water dHf within 1e-4 of MOPAC's -57.78934.
    z, xyz = harness.parse_lines(["O 0.000000 0.000000 0.000000", "H 0.960000 0.000000 0.000000",
                                  "H -0.240000 0.930000 0.000000"])
    r = harness.run(z, xyz)
    assert r["converged"] and r["iterations"] > 1
    assert abs(r["heat_of_formation_kcal"] - (-57.78934)) < 0.5  # geometry differs slightly from the unit test's


def test_nonconvergence_is_an_error():
    # src/scf.rs:770-775: a non-converged SCF is an error with no result.
    z, xyz = harness.parse_lines(["C 0 0 0", "H 1.09 0 0", "H -0.36 1.03 0", "H -0.36 -0.51 0.89",
                                  "H -0.36 -0.51 -0.89"])
    with pytest.raises(harness.OracleError) as info:
        harness.run(z, xyz, max_scf=1)
    assert info.value.code == 6


def test_invalid_inputs():
    z, xyz = harness.parse_lines(["H 0 0 0", "H 0 0 0"])
    with pytest.raises(harness.OracleError) as info:
        harness.run(z, xyz)
    assert info.value.code == 1
    z, xyz = harness.parse_lines(["H 0 0 0"])
    with pytest.raises(harness.OracleError):
        harness.run(z, xyz, multiplicity=2, reference="rhf")
    with pytest.raises(harness.OracleError):
        harness.run(z, xyz, multiplicity=1)  # one electron cannot be a singlet


def test_element_derivations():
    # src/params.rs:455-470 and src/mndod.rs:760-784: reference unit-test facts.
    c = harness.element(6)
    assert c[0] == 4
    s = harness.element(16)
    assert s[0] == 9
    rho0, rho1, rho2, dd = s[6], s[7], s[8], s[4]
    po = s[9:18]
    assert abs(po[0] - rho0) < 1e-12 and abs(po[1] - rho1) < 1e-12 and abs(po[2] - rho2) < 1e-12
    ddp = s[18:23]
    assert abs(ddp[0] - dd) < 1e-12
    assert s[23] == 0.0  # main-group eiscor
    fe = harness.element(26)
    assert abs(fe[23]) > 1.0
