"""Python host API of the engine: `run_pm7` and the stage functions over the C ABI.

Mirrors the reference's public surface for the molecular single point
(pm7-rs src/scf.rs:512-522 `run_pm7`, `Pm7Options` defaults :207-233, `Pm7Result`
fields :261-342): positions in Bohr, energies in eV, heat of formation in kcal/mol.
Errors raise `Pm7Error` carrying the C status code. There is no CPU fallback: when the
shared library or a CUDA device is missing the calls fail loudly.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "libpm7b200.so"

_lib = None

EXPORTED = [
    "pm7_params_load", "pm7_options_default", "pm7_run", "pm7_result_free", "pm7_last_error_message",
    "pm7_device_count", "pm7_stage_core_hamiltonian", "pm7_stage_fock", "pm7_stage_pair", "pm7_stage_core_core",
    "pm7_stage_corrections", "pm7_run_batch", "pm7_engine_config_default", "pm7_engine_create", "pm7_engine_submit",
    "pm7_engine_poll", "pm7_engine_destroy", "pm7_batch_partition", "pm7_stage_eigenvalues",
    "pm7_stage_product_tf32", "pm7_autotune_report", "pm7_gradient", "pm7_fixed_density_gradient",
    "pm7_correction_gradient", "pm7_run_batch_gradient", "pm7_engine_submit_gradient",
    "pm7_dandc_options_default", "pm7_run_dandc", "pm7_dandc_result_free", "pm7_stage_dandc_partition",
    "pm7_dandc_abi_sizes", "pm7_stage_seqsum", "pm7_stage_tf32_wait_drill",
    "pm7_engine_stats", "pm7_stage_fock_fp32", "pm7_stage_sp2_step_i8",
]


class Pm7Error(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code
        self.message = message

    def __reduce__(self):
        # results travel between ranks by pickling (host-side gather of a sharded batch)
        return (Pm7Error, (self.code, self.message))


def lib():
    """Load the engine's shared library (built in-tree by `make -C pm7-rs_b200`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is not built; run `make -C pm7-rs_b200`")
    L = C.CDLL(str(LIB_PATH))
    L.pm7_params_load.argtypes = [C.c_int32, C.POINTER(C.c_void_p)]
    L.pm7_options_default.argtypes = [C.POINTER(abi.Options)]
    L.pm7_run.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.POINTER(abi.Options), C.POINTER(abi.Result)]
    L.pm7_result_free.argtypes = [C.POINTER(abi.Result)]
    L.pm7_last_error_message.restype = C.c_char_p
    L.pm7_device_count.restype = C.c_int32
    L.pm7_stage_core_hamiltonian.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.c_int32, abi.DP,
                                             C.POINTER(C.c_int32)]
    L.pm7_stage_fock.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.c_int32, abi.DP, abi.DP, abi.DP]
    L.pm7_stage_fock_fp32.argtypes = L.pm7_stage_fock.argtypes
    L.pm7_stage_pair.argtypes = [C.c_void_p, C.c_int32, C.c_int32, abi.DP, C.c_int32, abi.DP, abi.DP, abi.DP, abi.DP,
                                 C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.pm7_stage_core_core.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, abi.DP]
    L.pm7_stage_corrections.argtypes = [C.POINTER(abi.Molecule), C.c_int32, C.c_int32, abi.DP]
    L.pm7_abi_sizes.argtypes = [C.POINTER(C.c_int64)]
    L.pm7_run_batch.argtypes = [C.c_int32, C.POINTER(abi.Molecule), C.c_void_p, C.POINTER(abi.Options),
                                C.POINTER(abi.Result), C.POINTER(C.c_int32)]
    L.pm7_batch_partition.argtypes = [C.c_int32, C.POINTER(abi.Molecule), C.c_int32, C.c_int32,
                                      C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.pm7_gradient.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.POINTER(abi.Options), C.POINTER(abi.Result),
                               abi.DP, abi.DP]
    L.pm7_fixed_density_gradient.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.c_int32, abi.DP, abi.DP, abi.DP]
    L.pm7_correction_gradient.argtypes = [C.POINTER(abi.Molecule), C.c_int32, C.c_int32, abi.DP]
    L.pm7_engine_submit_gradient.argtypes = [C.c_void_p, C.POINTER(abi.Molecule), C.POINTER(abi.Options), abi.DP,
                                             C.POINTER(C.c_uint64)]
    L.pm7_run_batch_gradient.argtypes = [C.c_int32, C.POINTER(abi.Molecule), C.c_void_p, C.POINTER(abi.Options),
                                         C.POINTER(abi.Result), C.POINTER(C.c_int32), C.POINTER(abi.DP)]
    L.pm7_dandc_options_default.argtypes = [C.POINTER(abi.DandcOptions)]
    L.pm7_run_dandc.argtypes = [C.POINTER(abi.Molecule), C.c_void_p, C.POINTER(abi.Options),
                                C.POINTER(abi.DandcOptions), C.c_int32, C.POINTER(abi.DandcResult)]
    L.pm7_dandc_result_free.argtypes = [C.POINTER(abi.DandcResult)]
    L.pm7_stage_dandc_partition.argtypes = [C.POINTER(abi.Molecule), C.c_int32, C.c_double, C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.pm7_stage_eigenvalues.argtypes = [C.c_int32, C.POINTER(C.c_int32), abi.DP, abi.DP, C.c_int32]
    L.pm7_stage_seqsum.argtypes = [C.c_int64, abi.DP, abi.DP, abi.DP, C.c_int32]
    L.pm7_stage_tf32_wait_drill.argtypes = [C.c_int32]
    L.pm7_engine_config_default.argtypes = [C.POINTER(abi.EngineConfig)]
    L.pm7_engine_create.argtypes = [C.POINTER(abi.EngineConfig), C.POINTER(C.c_void_p)]
    L.pm7_engine_submit.argtypes = [C.c_void_p, C.POINTER(abi.Molecule), C.POINTER(abi.Options),
                                    C.POINTER(C.c_uint64)]
    L.pm7_engine_poll.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(C.c_int32), C.POINTER(abi.Result),
                                  C.POINTER(C.c_double)]
    L.pm7_engine_destroy.argtypes = [C.c_void_p]
    L.pm7_engine_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    _lib = L
    return L


def device_count():
    return int(lib().pm7_device_count())


def _check(code):
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())


def params(method=0):
    """`Pm7Parameters::method` (src/params.rs:127-129): the cached parameter handle."""
    if isinstance(method, str):
        method = abi.METHODS[method]
    h = C.c_void_p()
    _check(lib().pm7_params_load(int(method), C.byref(h)))
    return h


class _Mol:
    def __init__(self, z, xyz_bohr):
        self.z = np.ascontiguousarray(z, dtype=np.uint8)
        self.xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
        if self.xyz.size != 3 * self.z.size:
            raise ValueError("xyz must hold 3 coordinates per atom")
        self.s = abi.Molecule(len(self.z), self.z.ctypes.data_as(C.POINTER(C.c_uint8)),
                              self.xyz.ctypes.data_as(abi.DP))


def _arr(ptr, n):
    if not ptr:
        return None
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def result_to_dict(r):
    n, nao = r.n_atoms, r.nao
    d = {k: getattr(r, k) for k in ("n_atoms", "nao", "n_occ", "n_occ_beta", "unrestricted", "iterations",
                                     "converged", "density_error", "electronic_ev", "core_ev", "total_ev",
                                     "heat_of_formation_kcal", "correction_kcal", "homo_ev", "lumo_ev",
                                     "homo_ev_beta", "lumo_ev_beta", "dipole_magnitude", "device_ms",
                                     "fp32_iterations")}
    for k in ("dipole_debye", "dipole_point_charge", "dipole_sp_hybrid", "dipole_pd_hybrid"):
        d[k] = np.array(list(getattr(r, k)))
    d["charges"] = _arr(r.charges, n)
    d["mo_energies"] = _arr(r.mo_energies, nao)
    d["mo_energies_beta"] = _arr(r.mo_energies_beta, nao)
    for k in ("density", "spin_density", "mo_coeff", "mo_coeff_beta"):
        a = _arr(getattr(r, k), nao * nao)
        d[k] = None if a is None else a.reshape(nao, nao)
    return d


def run_pm7(z, xyz_bohr, **options):
    """`run_pm7` (src/scf.rs:512-522) on the device. Options take the `Pm7Options`
    field names; the method may be given as a string ("pm7", "pm7-ts", ...)."""
    m = _Mol(z, xyz_bohr)
    keep = []
    for k in ("initial_density", "initial_spin_density"):
        if options.get(k) is not None:
            a = np.ascontiguousarray(options[k], dtype=np.float64)
            keep.append(a)
            options[k] = a.ctypes.data_as(abi.DP)
    o = abi.default_options(**options)
    h = params(o.method)
    r = abi.Result()
    code = lib().pm7_run(C.byref(m.s), h, C.byref(o), C.byref(r))
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())
    try:
        return result_to_dict(r)
    finally:
        lib().pm7_result_free(C.byref(r))


def closed_form_gradient(z, xyz_bohr, **options):
    """`closed_form_gradient` (src/gradient.rs:500-561) on the device: the SCF of `run_pm7`
    and the gradient of its total energy in eV/Bohr. Returns the fields of the reference's
    `GradientResult`: scf (the result dict), energy_ev, gradient (N x 3), forces (= -gradient)
    and max_gradient."""
    m = _Mol(z, xyz_bohr)
    keep = []
    for k in ("initial_density", "initial_spin_density"):
        if options.get(k) is not None:
            a = np.ascontiguousarray(options[k], dtype=np.float64)
            keep.append(a)
            options[k] = a.ctypes.data_as(abi.DP)
    o = abi.default_options(**options)
    h = params(o.method)
    r = abi.Result()
    g = np.zeros((len(m.z), 3))
    mx = C.c_double()
    code = lib().pm7_gradient(C.byref(m.s), h, C.byref(o), C.byref(r), g.ctypes.data_as(abi.DP), C.byref(mx))
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())
    try:
        scf = result_to_dict(r)
    finally:
        lib().pm7_result_free(C.byref(r))
    return {"scf": scf, "energy_ev": scf["total_ev"], "gradient": g, "forces": -g, "max_gradient": mx.value}


def dandc_result_to_dict(r):
    n, nao = r.n_atoms, r.nao
    d = {k: getattr(r, k) for k in ("n_atoms", "nao", "converged", "iterations", "subsystems", "largest_subsystem",
                                     "unrestricted", "fermi_ev", "electronic_ev", "density_error", "core_core_ev",
                                     "correction_ev", "energy_ev", "stored_density_elements")}
    d["converged"] = bool(d["converged"])
    d["unrestricted"] = bool(d["unrestricted"])
    d["charges"] = _arr(r.charges, n)
    g = _arr(r.gradient, 3 * n)
    d["gradient"] = None if g is None else g.reshape(n, 3)
    for k in ("density", "spin_density"):
        a = _arr(getattr(r, k), nao * nao)
        d[k] = None if a is None else a.reshape(nao, nao)
    return d


def run_dandc(z, xyz_bohr, dandc=None, gradient=True, **options):
    """`run_dandc` (src/dandc/mod.rs:143-428) and, with `gradient`, `dandc_derivatives`
    (:446-506) on the device. `dandc` holds `DandcOptions` fields (buffer in Bohr, core_size,
    fermi_width_ev, max_scf, p_tol, mixing); `options` the `Pm7Options` fields. Returns the
    `DandcResult` fields plus energy_ev, charges, the gradient (N x 3, eV/Bohr) and, when
    want_matrices is set, the dense global density (zeros outside the stored pattern). A run
    that reaches max_scf returns converged = False, as the reference does."""
    m = _Mol(z, xyz_bohr)
    o = abi.default_options(**options)
    d = abi.default_dandc_options(**(dandc or {}))
    r = abi.DandcResult()
    code = lib().pm7_run_dandc(C.byref(m.s), params(o.method), C.byref(o), C.byref(d), int(bool(gradient)),
                               C.byref(r))
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())
    try:
        return dandc_result_to_dict(r)
    finally:
        lib().pm7_dandc_result_free(C.byref(r))


def dandc_partition(z, xyz_bohr, core_size=12, buffer=15.0):
    """The subsystem partition `pm7_run_dandc` uses (host only): (core_of per atom, sizes per
    subsystem, stored atom pairs)."""
    m = _Mol(z, xyz_bohr)
    n = len(m.z)
    core_of = np.zeros(n, dtype=np.int32)
    sizes = np.zeros(max(n, 1), dtype=np.int32)
    count = C.c_int32()
    pairs = C.c_int64()
    _check(lib().pm7_stage_dandc_partition(C.byref(m.s), int(core_size), float(buffer),
                                           core_of.ctypes.data_as(C.POINTER(C.c_int32)),
                                           sizes.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(count),
                                           C.byref(pairs)))
    return core_of, sizes[:count.value].copy(), pairs.value


def dandc(z, xyz_bohr, buffer_angstrom=8.0, core_size=12, method="pm7", charge=0.0, multiplicity=1,
          reference="auto", scf_tolerance=None, max_scf=None):
    """The reference's Python `dandc` binding (src/python.rs:1409-1494): buffer in Angstrom
    (positions stay in Bohr, as everywhere in this API),
    raises when the SCF does not converge; returns energy_ev, energy_hartree,
    forces_ev_per_angstrom, fermi_ev, subsystems, largest_subsystem, iterations, unrestricted,
    stored_density_elements."""
    dc = {"buffer": buffer_angstrom * abi.ANGSTROM_TO_BOHR, "core_size": int(core_size),
          "max_scf": 200 if max_scf is None else int(max_scf),
          "p_tol": 1.0e-6 if scf_tolerance is None else float(scf_tolerance)}
    r = run_dandc(z, xyz_bohr, dandc=dc, gradient=True, method=method, charge=charge, multiplicity=multiplicity,
                  reference=reference, want_matrices=0)
    if not r["converged"]:
        raise ValueError(f"the divide-and-conquer SCF did not converge after {r['iterations']} iterations "
                         f"(error={r['density_error']:.3e})")
    return {"energy_ev": r["energy_ev"], "energy_hartree": r["energy_ev"] * abi.EV_TO_HARTREE,
            "forces_ev_per_angstrom": -r["gradient"] * abi.ANGSTROM_TO_BOHR, "fermi_ev": r["fermi_ev"],
            "subsystems": r["subsystems"], "largest_subsystem": r["largest_subsystem"],
            "iterations": r["iterations"], "unrestricted": r["unrestricted"],
            "stored_density_elements": r["stored_density_elements"]}


def fixed_density_gradient(z, xyz_bohr, p_total, p_spin=None, method=0, force_dpath=False):
    """`fixed_density_gradient_with` (src/gradient.rs:638-700), or with a spin density
    (P_alpha - P_beta) the UHF form (:1263-1350): core-core + electronic gradient, eV/Bohr."""
    m = _Mol(z, xyz_bohr)
    pt = np.ascontiguousarray(p_total, dtype=np.float64)
    ps = None if p_spin is None else np.ascontiguousarray(p_spin, dtype=np.float64)
    g = np.zeros((len(m.z), 3))
    _check(lib().pm7_fixed_density_gradient(C.byref(m.s), params(method), int(force_dpath), pt.ctypes.data_as(abi.DP),
                                            None if ps is None else ps.ctypes.data_as(abi.DP),
                                            g.ctypes.data_as(abi.DP)))
    return g


def correction_gradient(z, xyz_bohr, method=0, smooth=False):
    """`correction_gradient` (src/gradient.rs:208-261): post-SCF correction gradient, eV/Bohr."""
    m = _Mol(z, xyz_bohr)
    g = np.zeros((len(m.z), 3))
    _check(lib().pm7_correction_gradient(C.byref(m.s), int(method), int(smooth), g.ctypes.data_as(abi.DP)))
    return g


def core_hamiltonian(z, xyz_bohr, method=0, force_dpath=False):
    m = _Mol(z, xyz_bohr)
    h = params(method)
    nao = C.c_int32()
    _check(lib().pm7_stage_core_hamiltonian(C.byref(m.s), h, int(force_dpath), None, C.byref(nao)))
    out = np.zeros((nao.value, nao.value))
    _check(lib().pm7_stage_core_hamiltonian(C.byref(m.s), h, int(force_dpath), out.ctypes.data_as(abi.DP),
                                            C.byref(nao)))
    return out


def fock(z, xyz_bohr, p_tot, p_spin, method=0, force_dpath=False, fp32=False):
    """F = H + J(p_tot) - K(p_spin); fp32=True gives the mixed-precision cycles' FP32 build."""
    m = _Mol(z, xyz_bohr)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    ps = np.ascontiguousarray(p_spin, dtype=np.float64)
    f = np.zeros_like(pt)
    entry = lib().pm7_stage_fock_fp32 if fp32 else lib().pm7_stage_fock
    _check(entry(C.byref(m.s), params(method), int(force_dpath), pt.ctypes.data_as(abi.DP),
                 ps.ctypes.data_as(abi.DP), f.ctypes.data_as(abi.DP)))
    return f


def pair(zi, zj, d, method=0, force_dpath=False):
    dd = np.ascontiguousarray(d, dtype=np.float64)
    w = np.zeros(45 * 45)
    e1b, e2a, s = np.zeros(81), np.zeros(81), np.zeros(81)
    npi, npj = C.c_int32(), C.c_int32()
    _check(lib().pm7_stage_pair(params(method), int(zi), int(zj), dd.ctypes.data_as(abi.DP), int(force_dpath),
                                w.ctypes.data_as(abi.DP), e1b.ctypes.data_as(abi.DP), e2a.ctypes.data_as(abi.DP),
                                s.ctypes.data_as(abi.DP), C.byref(npi), C.byref(npj)))
    return (w[: npi.value * npj.value].reshape(npi.value, npj.value), e1b.reshape(9, 9), e2a.reshape(9, 9),
            s.reshape(9, 9))


def core_core(z, xyz_bohr, method=0):
    m = _Mol(z, xyz_bohr)
    e = C.c_double()
    _check(lib().pm7_stage_core_core(C.byref(m.s), params(method), C.byref(e)))
    return e.value


def tf32_wait_drill(n=128):
    """Status code of the bounded-wait drill (pm7_stage_tf32_wait_drill): the tcgen05
    squaring with its copies withheld; 10 (PM7_ERR_TIMEOUT) when every wait gave up."""
    return int(lib().pm7_stage_tf32_wait_drill(int(n)))


def seqsum(a, b=None, device=0):
    """The left-to-right f64 sum of a (or of the rounded products a*b), evaluated on the
    device with the exact bits of a serial loop: the fold the reference's energies use
    (`Matrix::frobenius_dot`, src/linalg.rs:138-141)."""
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
    if bb is not None and bb.size != a.size:
        raise ValueError("seqsum: a and b differ in length")
    out = C.c_double()
    _check(lib().pm7_stage_seqsum(a.size, a.ctypes.data_as(abi.DP), None if bb is None else bb.ctypes.data_as(abi.DP),
                                  C.byref(out), int(device)))
    return out.value


def corrections(z, xyz_bohr, method=0, smooth=False):
    m = _Mol(z, xyz_bohr)
    out = np.zeros(5)
    _check(lib().pm7_stage_corrections(C.byref(m.s), int(method), int(smooth), out.ctypes.data_as(abi.DP)))
    return out


def abi_sizes():
    out = (C.c_int64 * 3)()
    lib().pm7_abi_sizes(out)
    return tuple(out)


def dandc_abi_sizes():
    out = (C.c_int64 * 2)()
    lib().pm7_dandc_abi_sizes(out)
    return tuple(out)


def autotune_report():
    """The autotuner's choices so far in this process ({"<device>|<key>": variant})."""
    import json

    L = lib()
    L.pm7_autotune_report.restype = C.c_char_p
    return json.loads(L.pm7_autotune_report().decode())


def launch_count():
    """Kernels launched by the engine since process start."""
    lib().pm7_launch_count.restype = C.c_int64
    return int(lib().pm7_launch_count())


def profile_enable(on=True):
    lib().pm7_profile_enable.argtypes = [C.c_int32]
    lib().pm7_profile_enable(1 if on else 0)


def profile_read():
    """{stage: (total_ms, calls)} recorded since profile_enable(True)."""
    L = lib()
    L.pm7_profile_count.restype = C.c_int32
    L.pm7_profile_entry.argtypes = [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    out = {}
    for i in range(L.pm7_profile_count()):
        name, ms, calls = C.c_char_p(), C.c_double(), C.c_int64()
        _check(L.pm7_profile_entry(i, C.byref(name), C.byref(ms), C.byref(calls)))
        out[name.value.decode()] = (ms.value, calls.value)
    return out


def _options_with_arrays(options, keep):
    options = dict(options)
    for k in ("initial_density", "initial_spin_density"):
        if options.get(k) is not None:
            a = np.ascontiguousarray(options[k], dtype=np.float64)
            keep.append(a)
            options[k] = a.ctypes.data_as(abi.DP)
    return abi.default_options(**options)


def run_batch(molecules, options=None, **common):
    """Solve many molecules in one batched device run (`pm7_run_batch`).

    `molecules` is a list of (z, xyz_bohr); `options` an optional list of per-molecule
    option dicts merged over `common`. Returns one entry per molecule: the result dict
    of `run_pm7`, or the `Pm7Error` that `run_pm7` would have raised for it.
    """
    n = len(molecules)
    mols = [_Mol(z, x) for z, x in molecules]
    keep = []
    opts = (abi.Options * max(n, 1))()
    for i in range(n):
        o = dict(common)
        if options is not None:
            o.update(options[i])
        opts[i] = _options_with_arrays(o, keep)
    ms = (abi.Molecule * max(n, 1))(*[m.s for m in mols])
    res = (abi.Result * max(n, 1))()
    st = (C.c_int32 * max(n, 1))()
    h = params(opts[0].method if n else 0)
    code = lib().pm7_run_batch(n, ms, h, opts, res, st)
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())
    out = []
    for i in range(n):
        if st[i] == 0:
            out.append(result_to_dict(res[i]))
        else:
            out.append(Pm7Error(st[i], "batched solve failed"))
        lib().pm7_result_free(C.byref(res[i]))
    return out


def run_batch_gradient(molecules, options=None, **common):
    """`run_batch` with every molecule's nuclear gradient (`pm7_run_batch_gradient`).

    Returns one entry per molecule: the dict of `closed_form_gradient` (scf, energy_ev,
    gradient (N x 3, eV/Bohr), forces, max_gradient), or the `Pm7Error` for it.
    """
    n = len(molecules)
    mols = [_Mol(z, x) for z, x in molecules]
    keep = []
    opts = (abi.Options * max(n, 1))()
    for i in range(n):
        o = dict(common)
        if options is not None:
            o.update(options[i])
        opts[i] = _options_with_arrays(o, keep)
    ms = (abi.Molecule * max(n, 1))(*[m.s for m in mols])
    res = (abi.Result * max(n, 1))()
    st = (C.c_int32 * max(n, 1))()
    grads = [np.zeros((len(m.z), 3)) for m in mols]
    gp = (abi.DP * max(n, 1))(*[g.ctypes.data_as(abi.DP) for g in grads])
    h = params(opts[0].method if n else 0)
    code = lib().pm7_run_batch_gradient(n, ms, h, opts, res, st, gp)
    if code != 0:
        raise Pm7Error(code, lib().pm7_last_error_message().decode())
    out = []
    for i in range(n):
        if st[i] == 0:
            scf = result_to_dict(res[i])
            g = grads[i]
            out.append({"scf": scf, "energy_ev": scf["total_ev"], "gradient": g, "forces": -g,
                        "max_gradient": float(np.max(np.abs(g))) if g.size else 0.0})
        else:
            out.append(Pm7Error(st[i], "batched solve failed"))
        lib().pm7_result_free(C.byref(res[i]))
    return out


def batch_partition(molecules, n_ranks, method=0):
    """Longest-processing-time split of a batch over `n_ranks` (`pm7_batch_partition`).

    Returns (rank_of, rank_cost): the rank of each molecule and the estimated cost each
    rank carries. Host only; needs no GPU.
    """
    n = len(molecules)
    mols = [_Mol(z, x) for z, x in molecules]
    ms = (abi.Molecule * max(n, 1))(*[m.s for m in mols])
    owner = (C.c_int32 * max(n, 1))()
    load = (C.c_double * max(int(n_ranks), 1))()
    _check(lib().pm7_batch_partition(n, ms, int(method), int(n_ranks), owner, load))
    return np.array(owner[:n], dtype=np.int32), np.array(load[:n_ranks])


class Engine:
    """The serving engine (`pm7_engine_*`): submit requests as they arrive, poll results.

    Requests are admitted by their HBM footprint and advanced together one SCF iteration
    per step on the device; each finished request reports its submit-to-finish latency.
    """

    def __init__(self, method=0, device=0, hbm_budget_mb=-1, max_active=0):
        if isinstance(method, str):
            method = abi.METHODS[method]
        cfg = abi.EngineConfig()
        lib().pm7_engine_config_default(C.byref(cfg))
        cfg.device, cfg.method, cfg.hbm_budget_mb, cfg.max_active = device, method, hbm_budget_mb, max_active
        self._h = C.c_void_p()
        _check(lib().pm7_engine_create(C.byref(cfg), C.byref(self._h)))
        self.method = method
        self._keep = {}

    def submit(self, z, xyz_bohr, gradient=False, **options):
        """Queue a request; with gradient=True the finished result also carries "gradient"
        (N x 3, eV/Bohr) and "forces" (`pm7_engine_submit_gradient`)."""
        m = _Mol(z, xyz_bohr)
        keep = [m]
        options.setdefault("method", self.method)
        o = _options_with_arrays(options, keep)
        t = C.c_uint64()
        if gradient:
            g = np.zeros((len(m.z), 3))
            keep.append(g)
            _check(lib().pm7_engine_submit_gradient(self._h, C.byref(m.s), C.byref(o), g.ctypes.data_as(abi.DP),
                                                    C.byref(t)))
        else:
            g = None
            _check(lib().pm7_engine_submit(self._h, C.byref(m.s), C.byref(o), C.byref(t)))
        self._keep[t.value] = (keep, g)
        return t.value

    def stats(self):
        """Admission record: requests admitted, the most resident at once, the most device
        bytes they held at once, and the HBM budget in bytes (`pm7_engine_stats`)."""
        out = (C.c_int64 * 4)()
        _check(lib().pm7_engine_stats(self._h, out))
        return {"admitted": out[0], "peak_active": out[1], "peak_bytes": out[2], "budget_bytes": out[3]}

    def poll(self, ticket, wait=False):
        """(done, result): result is the run_pm7 dict plus "latency_ms", or a Pm7Error."""
        done = C.c_int32()
        r = abi.Result()
        lat = C.c_double()
        code = lib().pm7_engine_poll(self._h, ticket, int(bool(wait)), C.byref(done), C.byref(r), C.byref(lat))
        if not done.value:
            if code != 0:
                raise Pm7Error(code, lib().pm7_last_error_message().decode())
            return False, None
        _, g = self._keep.pop(ticket, (None, None))
        if code != 0:
            lib().pm7_result_free(C.byref(r))
            return True, Pm7Error(code, lib().pm7_last_error_message().decode())
        try:
            d = result_to_dict(r)
        finally:
            lib().pm7_result_free(C.byref(r))
        d["latency_ms"] = lat.value
        if g is not None:
            d["gradient"] = g
            d["forces"] = -g
        return True, d

    def close(self):
        if self._h:
            lib().pm7_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def eigenvalues(matrices, device=0):
    """Ascending eigenvalues of symmetric matrices on the GPU (`pm7_stage_eigenvalues`).

    `matrices` is a list of square arrays; returns one array of eigenvalues per matrix.
    """
    mats = [np.ascontiguousarray(m, dtype=np.float64) for m in matrices]
    orders = np.array([m.shape[0] for m in mats], dtype=np.int32)
    packed = np.concatenate([m.reshape(-1) for m in mats]) if mats else np.zeros(1)
    out = np.zeros(max(int(orders.sum()), 1))
    _check(lib().pm7_stage_eigenvalues(len(mats), orders.ctypes.data_as(C.POINTER(C.c_int32)),
                                       packed.ctypes.data_as(abi.DP), out.ctypes.data_as(abi.DP), int(device)))
    res, off = [], 0
    for n in orders:
        res.append(out[off:off + n].copy())
        off += n
    return res


def sp2_step_i8(x, square=True):
    """One fused FP64-accuracy SP2 step on the tcgen05 integer tensor cores (int8 digit
    planes): (x x or 2 x - x x, [tr, |.|_F^2] of it from the step's partials)."""
    L = lib()
    L.pm7_stage_sp2_step_i8.argtypes = [C.c_int32, abi.DP, C.c_int32, abi.DP, abi.DP]
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    out = np.zeros((n, n))
    norms = np.zeros(2)
    _check(L.pm7_stage_sp2_step_i8(n, x.ctypes.data_as(abi.DP), int(bool(square)), out.ctypes.data_as(abi.DP),
                                   norms.ctypes.data_as(abi.DP)))
    return out, norms


def product_tf32(a, b):
    """C = A B of two symmetric matrices on the tcgen05 tensor cores (3xTF32 split, fp32
    accumulation): the commutator product of the mixed-precision fp32 cycles."""
    L = lib()
    L.pm7_stage_product_tf32.argtypes = [C.c_int32, abi.DP, abi.DP, abi.DP]
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = a.shape[0]
    out = np.zeros((n, n))
    _check(L.pm7_stage_product_tf32(n, a.ctypes.data_as(abi.DP), b.ctypes.data_as(abi.DP), out.ctypes.data_as(abi.DP)))
    return out


def square_tf32(x):
    """C = X X of a symmetric matrix on the tcgen05 tensor cores (3xTF32 split, fp32
    accumulation): the squaring of the mixed-precision SP2 purification."""
    L = lib()
    L.pm7_stage_square_tf32.argtypes = [C.c_int32, abi.DP, abi.DP]
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    out = np.zeros((n, n))
    _check(L.pm7_stage_square_tf32(n, x.ctypes.data_as(abi.DP), out.ctypes.data_as(abi.DP)))
    return out
