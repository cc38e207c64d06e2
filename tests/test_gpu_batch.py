"""The batched and served device SCF against the single-molecule path and the oracle.

`pm7_run_batch` and the `pm7_engine_*` serving loop advance many closed-shell RHF
molecules together (one launch per SCF phase over all of them, per-molecule DIIS and
convergence control on the device). Each molecule's result must be the one `run_pm7`
gives for it: 1e-5 kcal/mol in the heat of formation against the oracle, and the same
result alone and in a mixed batch.
"""
import numpy as np
import pytest

from oracle import harness
from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu

DHF_TOL = 1.0e-5
Q_TOL = 1.0e-6


def _closed_shell_golden(golden, limit=None):
    out = []
    for name, case in sorted(golden.items()):
        if case["multiplicity"] != 1:
            continue
        z, x = harness.parse_lines(case["atoms"])
        out.append((name, z, x, float(case["charge"])))
    return out[:limit] if limit else out


def _mixed_set(golden):
    mols = [(n, z, x, q) for n, z, x, q in _closed_shell_golden(golden)]
    for k in (3, 9, 17):
        z, x = G.water_cluster(k, seed=k)
        mols.append((f"water{k}", z, x, 0.0))
    for n in (1, 5, 12, 23):
        z, x = G.alkane(n, seed=n)
        mols.append((f"alkane{n}", z, x, 0.0))
    return mols


def test_batch_matches_oracle_and_single_path(golden):
    mols = _mixed_set(golden)
    res = api.run_batch([(z, x) for _, z, x, _ in mols], options=[{"charge": q} for *_, q in mols])
    bad = []
    for (name, z, x, q), r in zip(mols, res):
        if isinstance(r, Exception):
            bad.append(f"{name}: {r}")
            continue
        o = harness.run(z, x, charge=q)
        if abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) > DHF_TOL:
            bad.append(f"{name}: dHf {r['heat_of_formation_kcal']} vs oracle {o['heat_of_formation_kcal']}")
        if np.max(np.abs(r["charges"] - o["charges"])) > Q_TOL:
            bad.append(f"{name}: charges")
        if abs(r["homo_ev"] - o["homo_ev"]) > 1e-5:
            bad.append(f"{name}: homo {r['homo_ev']} vs {o['homo_ev']}")
        np.testing.assert_allclose(r["dipole_debye"], o["dipole_debye"], rtol=0, atol=1e-5)
    assert not bad, "\n".join(bad)
    # the golden values themselves
    for (name, z, x, q), r in zip(mols, res):
        if name in golden:
            assert abs(r["heat_of_formation_kcal"] - golden[name]["pm7_rs"]["heat_of_formation_kcal"]) < DHF_TOL, name


def test_batch_statuses_mirror_run_pm7(golden):
    z_ok, x_ok = G.decane(1)
    z_rad, x_rad = harness.parse_lines(golden["methyl_radical"]["atoms"])
    mols = [(z_ok, x_ok), (np.array([1, 1], np.uint8), np.zeros((2, 3))), (z_rad, x_rad), (z_ok, x_ok)]
    opts = [{}, {}, {"multiplicity": 2}, {"max_scf": 2}]
    res = api.run_batch(mols, options=opts)
    assert not isinstance(res[0], Exception)
    assert isinstance(res[1], api.Pm7Error) and res[1].code == 1          # coincident atoms
    assert not isinstance(res[2], Exception) and res[2]["unrestricted"] == 1  # open shell: pm7_run path
    o = harness.run(z_rad, x_rad, multiplicity=2)
    assert abs(res[2]["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL
    assert isinstance(res[3], api.Pm7Error) and res[3].code == 6          # not converged in 2 cycles
    single = api.run_pm7(z_ok, x_ok)
    assert abs(res[0]["heat_of_formation_kcal"] - single["heat_of_formation_kcal"]) < 1e-7


def test_batch_matrices_are_consistent():
    z, x = G.water_cluster(6, seed=4)
    (r,) = api.run_batch([(z, x)], want_matrices=1)
    c = r["mo_coeff"]
    n_occ = r["n_occ"]
    p = 2.0 * c[:, :n_occ] @ c[:, :n_occ].T
    assert np.max(np.abs(p - r["density"])) < 1e-6
    s = api.run_pm7(z, x, want_matrices=1)
    assert np.max(np.abs(s["density"] - r["density"])) < 1e-6
    np.testing.assert_allclose(r["mo_energies"], s["mo_energies"], rtol=0, atol=1e-5)


def test_batch_options_level_shift_and_accelerators():
    z, x = G.alkane(4, seed=3)
    for kw in ({"accelerator": 0}, {"accelerator": 1}, {"level_shift": 0.5}):
        (r,) = api.run_batch([(z, x)], **kw)
        o = harness.run(z, x, **kw)
        assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL, kw


def test_engine_serves_and_alone_equals_mixed(golden):
    target = G.water_cluster(12, seed=21)
    others = [G.alkane(n, seed=n) for n in (2, 7, 15, 30)] + [G.water_cluster(k, seed=k) for k in (4, 20, 33)]
    with api.Engine() as eng:
        t = eng.submit(*target)
        done, alone = eng.poll(t, wait=True)
        assert done and not isinstance(alone, Exception)
        tickets = [eng.submit(*m) for m in others[:3]]
        t2 = eng.submit(*target)
        tickets += [eng.submit(*m) for m in others[3:]]
        done, mixed = eng.poll(t2, wait=True)
        assert done
        rest = [eng.poll(tk, wait=True)[1] for tk in tickets]
    assert all(not isinstance(r, Exception) for r in rest)
    assert mixed["latency_ms"] > 0
    # the same molecule alone and among others: identical to SCF precision
    assert abs(alone["heat_of_formation_kcal"] - mixed["heat_of_formation_kcal"]) < 1e-9
    assert alone["iterations"] == mixed["iterations"]
    assert np.max(np.abs(alone["charges"] - mixed["charges"])) < 1e-10
    o = harness.run(*target)
    assert abs(mixed["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL


def test_engine_serves_open_shells_beside_the_batch_and_rejects_bad_input():
    # open-shell (UHF) requests run through the single-molecule path on the engine's second
    # worker, beside closed-shell requests in the batch; results as run_pm7 / the oracle
    methyl = (np.array([6, 1, 1, 1], np.uint8), np.array([[0, 0, 0], [2.0, 0, 0], [-1.0, 1.7, 0], [-1.0, -1.7, 0]]))
    triplet_pair = (np.array([8, 8], np.uint8), np.array([[0, 0, 0], [1.21 / 0.529177210903, 0, 0]]))  # O2
    closed = [G.water_cluster(k, seed=k) for k in (3, 9)]
    with api.Engine() as eng:
        t1 = eng.submit(*methyl, multiplicity=2)
        tc = [eng.submit(*m) for m in closed]
        t2 = eng.submit(*triplet_pair, multiplicity=3)
        t3 = eng.submit(*methyl, multiplicity=2, gradient=True)
        r1, r2, r3 = (eng.poll(t, wait=True)[1] for t in (t1, t2, t3))
        rc = [eng.poll(t, wait=True)[1] for t in tc]
        t = eng.submit(np.array([1, 1], np.uint8), np.zeros((2, 3)))
        done, bad = eng.poll(t, wait=True)
        assert done and isinstance(bad, api.Pm7Error) and bad.code == 1
    for r, (z, x), mult in ((r1, methyl, 2), (r2, triplet_pair, 3), (r3, methyl, 2)):
        assert not isinstance(r, Exception) and r["unrestricted"]
        o = harness.run(z, x, multiplicity=mult)
        assert abs(r["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL
        assert np.max(np.abs(r["charges"] - o["charges"])) < Q_TOL
    single = api.closed_form_gradient(*methyl, multiplicity=2)
    np.testing.assert_allclose(r3["gradient"], single["gradient"], rtol=0, atol=1e-9)
    for r, m in zip(rc, closed):
        assert abs(r["heat_of_formation_kcal"] - harness.run(*m)["heat_of_formation_kcal"]) < DHF_TOL


def test_batch_density_by_sp2_and_by_eigensolver_agree(monkeypatch):
    # SP2 purification (tensor-core squarings) and the eigensolver give the same SCF
    mols = [G.water_cluster(k, seed=k) for k in (2, 11, 40)] + [G.alkane(n, seed=n) for n in (3, 18, 40)]
    monkeypatch.setenv("PM7_BATCH_DENSITY", "sp2")
    sp2 = api.run_batch(mols)
    monkeypatch.setenv("PM7_BATCH_DENSITY", "eig")
    eig = api.run_batch(mols)
    for a, b in zip(sp2, eig):
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1e-7
        assert np.max(np.abs(a["charges"] - b["charges"])) < 1e-8
        assert abs(a["homo_ev"] - b["homo_ev"]) < 1e-7


def test_batch_takes_the_single_path_iterations(golden):
    # the device-side DIIS of the batch follows the same trajectory as run_pm7
    for name in ("alkane_c20", "formic_acid_dimer", "benzene"):
        z, x = harness.parse_lines(golden[name]["atoms"])
        (r,) = api.run_batch([(z, x)])
        s = api.run_pm7(z, x)
        assert abs(r["iterations"] - s["iterations"]) <= 1, (name, r["iterations"], s["iterations"])


def test_batch_mixed_precision_within_tolerance():
    # fp32 purification cycles on the grouped tcgen05 squaring, fp64 cycles to finish:
    # heat of formation within 1e-4 kcal/mol of the fp64 batch, charges within 1e-5 e
    mols = [G.water_cluster(k, seed=k) for k in (20, 45, 64)] + [G.alkane(n, seed=n) for n in (17, 30, 40)]
    mols += [G.water_cluster(5, seed=1), G.alkane(3, seed=2)]  # below the SP2 size: unaffected
    f64 = api.run_batch(mols)
    mix = api.run_batch(mols, precision=1)
    for i, (a, b) in enumerate(zip(f64, mix)):
        assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1.0e-4, i
        assert np.max(np.abs(a["charges"] - b["charges"])) < 1.0e-5, i
    assert all(b["fp32_iterations"] > 0 for b in mix[:6])
    assert all(b["fp32_iterations"] == 0 for b in mix[6:])
    z, x = mols[2]
    o = harness.run(z, x)
    assert abs(mix[2]["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < 1.0e-4


def test_mixed_precision_large_chain_leaves_the_fp32_phase():
    # a 300+-atom S/Cl chain: the commutator norm stalls at the fp32 floor while the density
    # step is already small; the switch to fp64 must still happen and the SCF converge
    rng = np.random.default_rng(5)
    z, x = G.substituted_chain(110, rng)
    f = api.run_pm7(z, x, want_matrices=0)
    (b,) = api.run_batch([(z, x)], want_matrices=0, precision=1)
    s = api.run_pm7(z, x, want_matrices=0, precision=1)
    for r in (b, s):
        assert 0 < r["fp32_iterations"] < r["iterations"]
        assert abs(r["heat_of_formation_kcal"] - f["heat_of_formation_kcal"]) < 1.0e-4


def test_engine_without_matrices_retires_asynchronously_and_alone_equals_mixed():
    # without returned matrices a retirement's eigenvalue solves run beside the next SCF
    # step and its outputs are gathered one step later; results must not change
    target = G.water_cluster(14, seed=5)
    big = G.water_cluster(180, seed=6)  # order 1,080: the cluster eigenvalue kernel beside the next step
    others = [G.alkane(n, seed=n) for n in (3, 11, 26)] + [G.water_cluster(k, seed=k) for k in (8, 40)] + [big]
    with api.Engine() as eng:
        t = eng.submit(*target, want_matrices=0)
        done, alone = eng.poll(t, wait=True)
        assert done and not isinstance(alone, Exception)
        tickets = [eng.submit(*m, want_matrices=0) for m in others[:3]]
        t2 = eng.submit(*target, want_matrices=0)
        tickets += [eng.submit(*m, want_matrices=0) for m in others[3:]]
        done, mixed = eng.poll(t2, wait=True)
        rest = [eng.poll(tk, wait=True)[1] for tk in tickets]
    assert all(not isinstance(r, Exception) for r in rest)
    assert abs(alone["heat_of_formation_kcal"] - mixed["heat_of_formation_kcal"]) < 1e-9
    np.testing.assert_array_equal(alone["mo_energies"], mixed["mo_energies"])
    o = harness.run(*target)
    assert abs(mixed["heat_of_formation_kcal"] - o["heat_of_formation_kcal"]) < DHF_TOL
    assert abs(mixed["homo_ev"] - o["homo_ev"]) < 1e-5 and abs(mixed["lumo_ev"] - o["lumo_ev"]) < 1e-5
    full = api.run_pm7(*big, want_matrices=1)
    np.testing.assert_allclose(rest[-1]["mo_energies"], full["mo_energies"], rtol=0, atol=1e-8)
    assert abs(rest[-1]["heat_of_formation_kcal"] - full["heat_of_formation_kcal"]) < 1e-7
