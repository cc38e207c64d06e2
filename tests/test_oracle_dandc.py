"""The divide-and-conquer oracle against the properties pm7-rs's own tests assert
(tests/dandc.rs, src/dandc/partition.rs tests), which are its pins: the reference records no
divide-and-conquer golden numbers. The strongest one is exactness: with a buffer wider than
the molecule every subsystem is the whole molecule, and the result must be the exact SCF's."""
import numpy as np
import pytest

from oracle import harness
from pm7b200 import geometry as G

OPTS = dict(e_tol=1.0e-11, p_tol=1.0e-9)  # tests/dandc.rs:83-89


def test_energy_converges_to_the_exact_scf_as_the_buffer_grows():
    # tests/dandc.rs:129-172
    z, x = G.flat_alkane(10)
    exact = harness.run(z, x, want_matrices=0, **OPTS)
    errors = []
    for b in (6.0, 10.0, 14.0, 20.0, 30.0):
        r = harness.run_dandc(z, x, dandc=dict(buffer=b, core_size=6, p_tol=1e-8, max_scf=400), want_matrices=0,
                              **OPTS)
        assert r["converged"], (b, r["density_error"])
        errors.append(abs(r["electronic_ev"] - exact["electronic_ev"]))
    assert errors[-1] < errors[0] and errors[-1] < 0.05, errors
    # a 30 Bohr buffer holds the whole chain in every subsystem: the exact SCF itself
    assert errors[-1] < 1e-8, errors


def test_whole_molecule_buffer_reproduces_the_exact_density_and_charges():
    z, x = G.flat_alkane(6)
    exact = harness.run(z, x, **OPTS)
    r = harness.run_dandc(z, x, dandc=dict(buffer=40.0, core_size=4, p_tol=1e-10, max_scf=400), **OPTS)
    assert r["converged"]
    assert r["subsystems"] > 1 and r["largest_subsystem"] == len(z)
    assert np.abs(r["density"] - exact["density"]).max() < 1e-7
    assert np.abs(r["charges"] - exact["charges"]).max() < 1e-7
    assert abs(r["energy_ev"] - exact["total_ev"]) < 1e-7


def test_the_density_is_stored_sparsely():
    # tests/dandc.rs:174-208
    fractions = []
    for n in (10, 20, 40):
        z, x = G.flat_alkane(n)
        r = harness.run_dandc(z, x, dandc=dict(buffer=10.0, core_size=6, max_scf=1), want_matrices=0, **OPTS)
        fractions.append(r["stored_density_elements"] / r["nao"] ** 2)
    assert all(b < a for a, b in zip(fractions, fractions[1:])), fractions
    assert fractions[-1] < 0.35, fractions


def test_the_subsystem_size_does_not_grow_with_the_system():
    # tests/dandc.rs:210-243
    sizes = []
    for n in (10, 20, 40, 80):
        z, x = G.flat_alkane(n)
        r = harness.run_dandc(z, x, dandc=dict(buffer=10.0, core_size=6, max_scf=1), want_matrices=0, **OPTS)
        sizes.append((r["subsystems"], r["largest_subsystem"]))
    assert all(l <= sizes[0][1] + 4 for _, l in sizes), sizes
    assert sizes[-1][0] >= 6 * sizes[0][0], sizes


def test_the_gradient_converges_to_the_exact_one_as_the_buffer_grows():
    # tests/dandc.rs:245-290
    z, x = G.flat_alkane(8)
    _, exact = harness.gradient(z, x, **OPTS)
    worst = []
    for b in (8.0, 14.0, 22.0, 34.0):
        r = harness.run_dandc(z, x, dandc=dict(buffer=b, core_size=6, p_tol=1e-8, max_scf=400), gradient=True,
                              **OPTS)
        worst.append(np.linalg.norm(r["gradient"] - exact, axis=1).max())
    assert worst[-1] < worst[0] and worst[-1] < 2.0e-3, worst


def ethyl():
    # tests/dandc.rs:409-417 (Angstrom)
    z = np.array([6, 6, 1, 1, 1], dtype=np.uint8)
    x = np.array([[0.0, 0.0, 0.0], [1.50, 0.0, 0.0], [-0.5, 0.9, 0.0], [-0.5, -0.9, 0.0], [2.05, 0.92, 0.0]])
    return z, x / 0.529177210903


def test_an_open_shell_system_runs_unrestricted():
    # tests/dandc.rs:408-436
    z, x = ethyl()
    r = harness.run_dandc(z, x, dandc=dict(buffer=25.0, core_size=3, max_scf=400, p_tol=1e-8), multiplicity=2,
                          **OPTS)
    assert r["unrestricted"] and r["converged"]
    nao = r["nao"]
    assert abs(np.trace(r["spin_density"]) - 1.0) < 0.15


def test_every_atom_is_the_core_of_exactly_one_subsystem_and_weights_cover_the_pattern():
    # partition.rs tests: a hydrogen chain at 2 Bohr spacing; the core counts partition the atoms
    n = 40
    z = np.ones(n, dtype=np.uint8)
    x = np.zeros((n, 3))
    x[:, 0] = 2.0 * np.arange(n)
    small = harness.run_dandc(z, x, dandc=dict(buffer=6.0, core_size=5, max_scf=1), charge=0.0, want_matrices=0,
                              **OPTS)
    big_z = np.ones(4 * n, dtype=np.uint8)
    big_x = np.zeros((4 * n, 3))
    big_x[:, 0] = 2.0 * np.arange(4 * n)
    large = harness.run_dandc(big_z, big_x, dandc=dict(buffer=6.0, core_size=5, max_scf=1), want_matrices=0, **OPTS)
    assert large["subsystems"] == 4 * small["subsystems"]
    assert large["largest_subsystem"] <= small["largest_subsystem"] + 1


@pytest.mark.parametrize("bad, text", [
    (dict(buffer=0.0), "buffer must be finite and positive"),
    (dict(buffer=float("nan")), "buffer must be finite and positive"),
    (dict(core_size=0), "core size must be at least 1"),
    (dict(fermi_width_ev=0.0), "Fermi width"),
    (dict(mixing=0.0), "mixing factor"),
    (dict(mixing=1.5), "mixing factor"),
])
def test_invalid_options_are_refused(bad, text):
    # src/dandc/mod.rs:83-110
    z, x = G.flat_alkane(2)
    with pytest.raises(harness.OracleError) as e:
        harness.run_dandc(z, x, dandc=bad)
    assert text in str(e.value)


def test_no_chemical_potential_is_an_error_naming_the_spectrum():
    # src/dandc/mod.rs:741-757: more electrons than the subsystem states hold
    z = np.array([1, 1], dtype=np.uint8)
    x = np.array([[0.0, 0.0, 0.0], [1.4, 0.0, 0.0]])
    with pytest.raises(harness.OracleError) as e:
        harness.run_dandc(z, x, dandc=dict(buffer=10.0, core_size=1), charge=-10.0)
    assert "no chemical potential" in str(e.value) and "spectra span" in str(e.value)
