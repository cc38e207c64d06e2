"""Divide-and-conquer SCF on the device (pm7_run_dandc) against the oracle's restatement of
pm7-rs run_dandc / dandc_derivatives, and against the exact SCF where the buffer holds the
whole molecule. Both sides stop when the RMS density change falls below p_tol, so they may
stop an iteration apart; the tolerances below allow for that and nothing more."""
import numpy as np
import pytest

from oracle import harness
from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu

OPTS = dict(e_tol=1.0e-11, p_tol=1.0e-9)


def _compare(d, o, e_tol=2e-6, p_tol=2e-6):
    for k in ("converged", "subsystems", "largest_subsystem", "unrestricted", "stored_density_elements", "nao"):
        assert d[k] == o[k], (k, d[k], o[k])
    assert abs(d["iterations"] - o["iterations"]) <= 2, (d["iterations"], o["iterations"])
    assert abs(d["electronic_ev"] - o["electronic_ev"]) < e_tol, (d["electronic_ev"], o["electronic_ev"])
    assert abs(d["energy_ev"] - o["energy_ev"]) < e_tol
    assert abs(d["core_core_ev"] - o["core_core_ev"]) < 1e-8 * max(1.0, abs(o["core_core_ev"]))
    assert abs(d["correction_ev"] - o["correction_ev"]) < 1e-9
    assert np.abs(d["charges"] - o["charges"]).max() < p_tol
    if o.get("density") is not None:
        assert np.abs(d["density"] - o["density"]).max() < p_tol
    if o.get("spin_density") is not None:
        assert np.abs(d["spin_density"] - o["spin_density"]).max() < p_tol


@pytest.mark.parametrize("buffer", [6.0, 10.0, 14.0, 20.0, 30.0])
def test_alkane_chain_matches_the_oracle(buffer):
    # the chain and buffers of pm7-rs tests/dandc.rs:129-172
    z, x = G.flat_alkane(10)
    dc = dict(buffer=buffer, core_size=6, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=False, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, **OPTS)
    _compare(d, o)


def test_whole_molecule_buffer_is_the_exact_scf():
    z, x = G.flat_alkane(10)
    exact = api.run_pm7(z, x, **OPTS)
    d = api.run_dandc(z, x, dandc=dict(buffer=40.0, core_size=6, p_tol=1e-10, max_scf=400), **OPTS)
    assert d["converged"] and d["largest_subsystem"] == len(z)
    assert abs(d["energy_ev"] - exact["total_ev"]) < 1e-7
    assert np.abs(d["density"] - exact["density"]).max() < 1e-7
    assert np.abs(d["charges"] - exact["charges"]).max() < 1e-7


def test_large_subsystems_take_the_per_matrix_solver_and_stay_exact():
    # 100 waters (nao 600): every subsystem holds the cluster, so each is solved at order
    # 640 by dsyevd instead of the batched solver
    z, x = G.water_cluster(100, seed=3)
    exact = api.run_pm7(z, x, want_matrices=0, e_tol=1e-10, p_tol=1e-8)
    d = api.run_dandc(z, x, dandc=dict(buffer=200.0, core_size=60, p_tol=1e-9, max_scf=400), gradient=False,
                      want_matrices=0)
    assert d["converged"] and d["subsystems"] > 1 and d["largest_subsystem"] == 300
    assert abs(d["energy_ev"] - exact["total_ev"]) < 1e-6
    assert np.abs(d["charges"] - exact["charges"]).max() < 1e-6


@pytest.mark.parametrize("method", [1, 3, 4])
def test_method_variants_match_the_oracle(method):
    # PM7-TS, PM7-minus (no corrections), PM7-HH (its H-H repulsion term)
    z, x = G.flat_alkane(8)
    dc = dict(buffer=10.0, core_size=6, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=False, method=method, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, method=method, **OPTS)
    _compare(d, o)


def test_smooth_dispersion_matches_the_oracle():
    z, x = G.water_cluster(12, seed=4)
    dc = dict(buffer=9.0, core_size=9, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=True, smooth_dispersion=1, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, gradient=True, smooth_dispersion=1, **OPTS)
    _compare(d, o)
    assert np.abs(d["gradient"] - o["gradient"]).max() < 1e-5 + 1e-6 * np.abs(o["gradient"]).max()


def test_water_cluster_matches_the_oracle():
    z, x = G.water_cluster(40, seed=1)
    dc = dict(buffer=10.0, core_size=12, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=False, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, **OPTS)
    _compare(d, o)


def test_d_shell_subsystems_match_the_oracle():
    rng = np.random.default_rng(5)
    z, x = G.substituted_chain(14, rng, p_s=0.3, p_cl=0.2)
    assert (z == 16).any() or (z == 17).any()
    dc = dict(buffer=9.0, core_size=6, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=False, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, **OPTS)
    _compare(d, o)


def test_open_shell_runs_unrestricted_like_the_oracle():
    from test_oracle_dandc import ethyl

    z, x = ethyl()
    dc = dict(buffer=25.0, core_size=3, max_scf=400, p_tol=1e-8)
    d = api.run_dandc(z, x, dandc=dc, multiplicity=2, gradient=False, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, multiplicity=2, **OPTS)
    _compare(d, o)
    assert abs(np.trace(d["spin_density"]) - 1.0) < 0.15


def test_open_shell_chain_with_small_buffer_matches_the_oracle():
    z, x = G.flat_alkane(7)
    dc = dict(buffer=9.0, core_size=5, max_scf=400, p_tol=1e-8)
    d = api.run_dandc(z, x, dandc=dc, multiplicity=3, gradient=False, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, multiplicity=3, **OPTS)
    _compare(d, o)


def test_gradient_matches_the_oracle():
    # dandc_derivatives (src/dandc/mod.rs:446-506) at a partial buffer
    z, x = G.flat_alkane(8)
    dc = dict(buffer=14.0, core_size=6, p_tol=1e-9, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=True, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, gradient=True, **OPTS)
    assert np.abs(d["gradient"] - o["gradient"]).max() < 1e-5 + 1e-6 * np.abs(o["gradient"]).max()


def test_gradient_converges_to_the_exact_one():
    # tests/dandc.rs:245-290 on the device
    z, x = G.flat_alkane(8)
    exact = api.closed_form_gradient(z, x, **OPTS)["gradient"]
    worst = []
    for b in (8.0, 14.0, 22.0, 34.0):
        d = api.run_dandc(z, x, dandc=dict(buffer=b, core_size=6, p_tol=1e-8, max_scf=400), want_matrices=0, **OPTS)
        worst.append(np.linalg.norm(d["gradient"] - exact, axis=1).max())
    assert worst[-1] < worst[0] and worst[-1] < 2.0e-3, worst


def test_python_binding_shape():
    z, x = G.flat_alkane(6)
    r = api.dandc(z, x, buffer_angstrom=8.0, core_size=6)
    for k in ("energy_ev", "energy_hartree", "forces_ev_per_angstrom", "fermi_ev", "subsystems", "largest_subsystem",
              "iterations", "unrestricted", "stored_density_elements"):
        assert k in r
    assert r["forces_ev_per_angstrom"].shape == (len(z), 3)
    with pytest.raises(ValueError):
        api.dandc(z, x, buffer_angstrom=8.0, core_size=6, max_scf=1)


def test_not_converged_is_reported_not_raised():
    z, x = G.flat_alkane(6)
    d = api.run_dandc(z, x, dandc=dict(buffer=8.0, core_size=4, max_scf=2), gradient=False)
    assert not d["converged"] and d["iterations"] == 2


@pytest.mark.parametrize("bad", [dict(buffer=0.0), dict(core_size=0), dict(fermi_width_ev=-1.0), dict(mixing=2.0)])
def test_invalid_options_are_refused(bad):
    z, x = G.flat_alkane(2)
    with pytest.raises(api.Pm7Error) as e:
        api.run_dandc(z, x, dandc=bad)
    assert e.value.code == 1


def test_memory_budget_names_the_buffer():
    z, x = G.flat_alkane(20)
    with pytest.raises(api.Pm7Error) as e:
        api.run_dandc(z, x, dandc=dict(buffer=30.0, core_size=6), max_memory_mb=1)
    assert e.value.code == 1 and "buffer" in e.value.message


def test_no_chemical_potential_is_an_error_naming_the_spectrum():
    z = np.array([1, 1], dtype=np.uint8)
    x = np.array([[0.0, 0.0, 0.0], [1.4, 0.0, 0.0]])
    with pytest.raises(api.Pm7Error) as e:
        api.run_dandc(z, x, dandc=dict(buffer=10.0, core_size=1), charge=-10.0)
    assert e.value.code == 1 and "no chemical potential" in e.value.message and "spectra span" in e.value.message


def test_single_atom_and_sparkle_free_edge_cases():
    z = np.array([8], dtype=np.uint8)
    x = np.zeros((1, 3))
    dc = dict(buffer=10.0, core_size=4, p_tol=1e-8, max_scf=400)
    d = api.run_dandc(z, x, dandc=dc, gradient=True, charge=-2.0, **OPTS)
    o = harness.run_dandc(z, x, dandc=dc, charge=-2.0, **OPTS)
    _compare(d, o)
    assert d["subsystems"] == 1 and np.abs(d["gradient"]).max() < 1e-12
