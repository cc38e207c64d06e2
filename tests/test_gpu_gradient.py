"""Device nuclear gradient (pm7_gradient, pm7_fixed_density_gradient, pm7_correction_gradient)
against the oracle.

The device differentiates each atom pair's fixed-density energy (and the correction energy)
by the five-point difference of its own integral kernels; the oracle differentiates the whole
fixed-density energy of its CPU restatement the same way (the reference's `analytic_gradient`
route), pinned by tests/test_oracle_gradient.py to the reference's gradient tests. At a shared
density the two agree to rounding (1e-6 eV/Bohr here); through each engine's own SCF they
agree to the SCF's convergence (1e-5 eV/Bohr).
"""
import numpy as np
import pytest

from oracle import harness as H
from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu

A0 = 0.529177210903
FIXED_TOL = 1.0e-6   # eV/Bohr, same density on both sides
SCF_TOL = 1.0e-5     # eV/Bohr, each side's own converged density
FD_TOL = 5.0e-5      # eV/Bohr, against full-SCF energy differences (src/gradient.rs:1552-1576)

# src/gradient.rs:1530,1555,1581,1608 (Angstrom)
SMALL = {
    "water": ([8, 1, 1], [[0.0, 0.0, 0.0], [1.02, 0.0, 0.0], [-0.28, 0.96, 0.0]], 1),
    "formaldehyde": ([6, 8, 1, 1], [[0.0, 0.0, 0.0], [0.03, 0.0, 1.25], [0.95, 0.02, -0.55], [-0.94, -0.03, -0.52]], 1),
    "h2s": ([16, 1, 1], [[0.0, 0.0, 0.0], [0.0, 0.9705, 0.9430], [0.0, -0.9705, 0.9430]], 1),
    "methyl": ([6, 1, 1, 1], [[0.0, 0.0, 0.05], [1.12, 0.0, 0.0], [-0.55, 0.95, 0.0], [-0.55, -0.95, 0.0]], 2),
}


def small(name):
    z, xyz, mult = SMALL[name]
    return np.array(z), np.array(xyz) / A0, mult


def chain_with_s_cl(n=12, seed=5):
    rng = np.random.default_rng(seed)
    for _ in range(50):
        z, x = G.substituted_chain(n, rng)
        if any(v in (16, 17) for v in z):
            return z, x
    raise AssertionError("no S/Cl drawn")


def ethyne_and_silanol():
    # H-C#C-H beside H3Si-O-H, 6 Angstrom apart: the C#C and Si-O-H correction terms
    atoms = [(1, (-1.66, 0.0, 0.0)), (6, (-0.60, 0.0, 0.0)), (6, (0.60, 0.0, 0.0)), (1, (1.66, 0.0, 0.0)),
             (14, (0.0, 6.0, 0.0)), (8, (1.64, 6.0, 0.0)), (1, (2.12, 6.83, 0.0)), (1, (-0.49, 7.39, 0.0)),
             (1, (-0.49, 5.30, 1.20)), (1, (-0.49, 5.30, -1.20))]
    z = np.array([a for a, _ in atoms])
    x = np.array([p for _, p in atoms]) / A0
    return z, x


def fixed_density_case(name):
    if name in SMALL:
        z, x, mult = small(name)
        return z, x, mult, False
    if name == "water20":
        z, x = G.water_cluster(20, seed=1)
        return z, x, 1, False
    if name == "water40":  # wider than the H-bond reach of one atom (8.4-9.4 A in water)
        z, x = G.water_cluster(40, seed=6)
        return z, x, 1, False
    if name == "chain_s_cl":
        z, x = chain_with_s_cl()
        return z, x, 1, False
    if name == "octane_dframe":
        z, x = G.alkane(8, seed=2)
        return z, x, 1, True
    raise KeyError(name)


@pytest.mark.parametrize("name", ["water", "formaldehyde", "h2s", "methyl", "water20", "chain_s_cl", "octane_dframe"])
def test_fixed_density_gradient_matches_oracle(name):
    z, x, mult, dpath = fixed_density_case(name)
    r = H.run(z, x, multiplicity=mult, force_dpath=dpath, want_matrices=1)
    ps = r["spin_density"] if r["unrestricted"] else None
    ref = H.fixed_density_gradient(z, x, r["density"], ps, force_dpath=dpath)
    got = api.fixed_density_gradient(z, x, r["density"], ps, force_dpath=dpath)
    assert np.max(np.abs(got - ref)) < FIXED_TOL, (name, np.max(np.abs(got - ref)))


@pytest.mark.parametrize("case,method,smooth", [("water20", 0, False), ("water40", 0, False), ("water20", 4, False),
                                                ("water20", 0, True), ("ethyne_silanol", 0, False),
                                                ("chain_s_cl", 0, False), ("water20", 3, False)])
def test_correction_gradient_matches_oracle(case, method, smooth):
    if case == "ethyne_silanol":
        z, x = ethyne_and_silanol()
    else:
        z, x, _, _ = fixed_density_case(case)
    ref = H.correction_gradient(z, x, method=method, smooth=smooth)
    got = api.correction_gradient(z, x, method=method, smooth=smooth)
    assert np.max(np.abs(got - ref)) < FIXED_TOL, (case, method, np.max(np.abs(got - ref)))
    if method == 3:
        assert np.all(got == 0.0)  # PM7-minus: no corrections


def test_correction_gradient_terms_present():
    # the H-bond, C#C and Si-O-H terms contribute (non-zero) gradients on these geometries
    z, x = ethyne_and_silanol()
    assert np.max(np.abs(api.correction_gradient(z, x))) > 1.0e-6
    z, x, _, _ = fixed_density_case("water20")
    assert np.max(np.abs(api.correction_gradient(z, x))) > 1.0e-4


@pytest.mark.parametrize("name", ["formaldehyde", "h2s", "methyl"])
def test_closed_form_gradient_matches_oracle(name):
    z, x, mult = small(name)
    out = api.closed_form_gradient(z, x, multiplicity=mult)
    r, ref = H.gradient(z, x, multiplicity=mult)
    assert abs(out["scf"]["total_ev"] - r["total_ev"]) < 1.0e-6
    assert np.max(np.abs(out["gradient"] - ref)) < SCF_TOL, (name, np.max(np.abs(out["gradient"] - ref)))
    assert np.array_equal(out["forces"], -out["gradient"])
    assert out["max_gradient"] == pytest.approx(np.max(np.abs(out["gradient"])), abs=0.0)
    assert out["energy_ev"] == out["scf"]["total_ev"]
    assert out["scf"]["unrestricted"] == (mult > 1)


def test_closed_form_gradient_cluster_with_corrections():
    z, x = G.water_cluster(8, seed=3)
    out = api.closed_form_gradient(z, x)
    _, ref = H.gradient(z, x)
    assert np.max(np.abs(out["gradient"] - ref)) < SCF_TOL


def test_gradient_matches_scf_energy_difference():
    # the reference's own check (src/gradient.rs:1552-1576), through the device SCF alone
    z, x, mult = small("formaldehyde")
    g = api.closed_form_gradient(z, x, multiplicity=mult)["gradient"]
    num = np.zeros_like(g)
    h = 1.0e-4
    for a in range(len(z)):
        for k in range(3):
            e = []
            for t in (h, -h):
                y = x.copy()
                y[a, k] += t
                e.append(api.run_pm7(z, y, multiplicity=mult, want_matrices=0)["total_ev"])
            num[a, k] = (e[0] - e[1]) / (2 * h)
    assert np.max(np.abs(g - num)) < FD_TOL, np.max(np.abs(g - num))


def test_gradient_invariances_300_atoms():
    # a 100-water cluster: the pair forces cancel in the sum (translation) and the torque is
    # bounded by the SCF's convergence (Hellmann-Feynman at the converged density)
    z, x = G.water_cluster(100, seed=4)
    out = api.closed_form_gradient(z, x, want_matrices=0)
    g = out["gradient"]
    assert np.all(np.isfinite(g))
    assert np.max(np.abs(g.sum(axis=0))) < 1.0e-6
    c = x - x.mean(axis=0)
    assert np.max(np.abs(np.cross(c, g).sum(axis=0))) < 1.0e-3


def test_gradient_errors_and_edge_cases():
    # one atom: no pairs, zero gradient; an open shell forced to RHF is an input error
    one = np.array([8]), np.zeros((1, 3))
    assert np.all(api.fixed_density_gradient(*one, np.diag([2.0, 4 / 3, 4 / 3, 4 / 3])) == 0.0)
    assert np.all(api.correction_gradient(*one) == 0.0)
    z, x, _ = small("water")
    with pytest.raises(api.Pm7Error):
        api.closed_form_gradient(z, x, multiplicity=2, reference=1)  # RHF with an open shell


def _break_aware(e, h):
    # the rule of the device and the oracle: five-point on a smooth stencil, else the one-sided
    # formula of the side without the break
    em2, em1, e0, ep1, ep2 = e
    d = [em1 - em2, e0 - em1, ep1 - e0, ep2 - ep1]
    t1, t2 = (d[2] - d[1]) - (d[1] - d[0]), (d[3] - d[2]) - (d[2] - d[1])
    if abs(t1) <= 1e-9 and abs(t2) <= 1e-9:
        return (8 * (ep1 - em1) - (ep2 - em2)) / (12 * h)
    sl, sr, sm = abs(d[1] - d[0]), abs(d[3] - d[2]), abs(d[2] - d[1])
    left, right = (3 * e0 - 4 * em1 + em2) / (2 * h), (-3 * e0 + 4 * ep1 - ep2) / (2 * h)
    if max(sl, sr) < 0.01 * sm:  # the break is at the point
        return right
    if sl < 0.5 * sr:
        return left
    if sr < 0.5 * sl:
        return right
    return (ep1 - em1) / (2 * h)


def test_correction_gradient_across_an_hbond_switch_3000_atoms():
    # In the 1,000-water cluster (seed 0) the EH+ energy jumps by 0.17 kcal/mol when O 1131
    # moves by +1.5e-5..2e-5 Bohr along x: inside the +2h point of the stencil. The gradient
    # must be the derivative of the branch the geometry is on (the oracle's correction energy,
    # evaluated at the five points, under the same rule), not the 60 eV/Bohr a plain five-point
    # difference gives; and the whole cluster's correction forces must still sum to zero.
    z, x = G.water_cluster(1000, seed=0)
    g = api.correction_gradient(z, x)
    h, a = 1.0e-5, 1131
    e = []
    for t in (-2, -1, 0, 1, 2):
        y = x.copy()
        y[a, 0] += t * h
        e.append(float(np.sum(H.corrections(z, y))))
    ref = _break_aware(e, h) / 23.06054783061903
    assert abs(g[a, 0] - ref) < FIXED_TOL, (g[a, 0], ref)
    assert abs(g[a, 0]) < 1.0
    assert np.max(np.abs(g.sum(axis=0))) < 1.0e-6


def test_batched_gradients_match_single():
    # pm7_run_batch_gradient: closed-shell molecules through the batch engine (gradient at the
    # density the batch converged to), the UHF radical through pm7_gradient; each must match
    # the single-molecule gradient to the SCF's convergence
    mols = [G.alkane(3, seed=1), G.water_cluster(6, seed=2), chain_with_s_cl(6, seed=8)]
    z, x, _ = small("methyl")
    mols.append((z, x))
    opts = [{}, {}, {}, {"multiplicity": 2}]
    out = api.run_batch_gradient(mols, options=opts)
    for (zz, xx), o, r in zip(mols, opts, out):
        assert not isinstance(r, Exception), r
        single = api.closed_form_gradient(zz, xx, **o)
        assert abs(r["scf"]["heat_of_formation_kcal"] - single["scf"]["heat_of_formation_kcal"]) < 1.0e-5
        assert np.max(np.abs(r["gradient"] - single["gradient"])) < SCF_TOL, np.max(np.abs(r["gradient"] - single["gradient"]))
        assert np.array_equal(r["forces"], -r["gradient"])


TM_CASES = ["ferrocene", "titanocene_dichloride", "chromyl_chloride", "permanganate", "tetrachloroplatinate",
            "copper_chloride", "nickel_tetracarbonyl"]


@pytest.mark.parametrize("name", TM_CASES)
def test_fixed_density_gradient_transition_metals(golden, name):
    # d-shell metals (PM7 d balance, 45x45 one-centre blocks) in the MNDO/d frame, at the
    # oracle's converged density for the reference's golden geometries
    case = golden[name]
    z, x = H.parse_lines(case["atoms"])
    r = H.run(z, x, charge=float(case["charge"]), multiplicity=case["multiplicity"], want_matrices=1)
    ps = r["spin_density"] if r["unrestricted"] else None
    ref = H.fixed_density_gradient(z, x, r["density"], ps)
    got = api.fixed_density_gradient(z, x, r["density"], ps)
    assert np.max(np.abs(got - ref)) < FIXED_TOL, (name, np.max(np.abs(got - ref)))


def test_closed_form_gradient_ferrocene(golden):
    case = golden["ferrocene"]
    z, x = H.parse_lines(case["atoms"])
    out = api.closed_form_gradient(z, x, charge=float(case["charge"]))
    _, ref = H.gradient(z, x, charge=float(case["charge"]))
    assert np.max(np.abs(out["gradient"] - ref)) < SCF_TOL


def test_served_gradients_match_single():
    # pm7_engine_submit_gradient: requests with and without a gradient in one serving engine
    mols = [G.alkane(4, seed=3), G.water_cluster(5, seed=4), chain_with_s_cl(5, seed=9)]
    with api.Engine() as eng:
        tickets = [eng.submit(z, x, gradient=True) for z, x in mols] + [eng.submit(*mols[0])]
        out = [eng.poll(t, wait=True)[1] for t in tickets]
    for (z, x), r in zip(mols, out[:3]):
        assert not isinstance(r, Exception), r
        single = api.closed_form_gradient(z, x)
        assert np.max(np.abs(r["gradient"] - single["gradient"])) < SCF_TOL
        assert np.array_equal(r["forces"], -r["gradient"])
    assert "gradient" not in out[3]
