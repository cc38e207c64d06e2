"""ctypes mirror of include/pm7_b200.h (the engine's C ABI).

Field order and types must match the header exactly; tests/test_abi.py checks the
struct sizes against the compiled library's own sizeof report.
"""
import ctypes as C

PM7_OK = 0
STATUS_NAMES = {
    0: "PM7_OK",
    1: "PM7_ERR_INVALID_INPUT",
    2: "PM7_ERR_MISSING_ELEMENT",
    3: "PM7_ERR_MISSING_PARAMETER",
    4: "PM7_ERR_UNSUPPORTED",
    5: "PM7_ERR_LINEAR_ALGEBRA",
    6: "PM7_ERR_SCF_NOT_CONVERGED",
    7: "PM7_ERR_RESPONSE_FAILED",
    8: "PM7_ERR_INSUFFICIENT_MEMORY",
    9: "PM7_ERR_CUDA",
    10: "PM7_ERR_TIMEOUT",
}

METHODS = {"pm7": 0, "pm7-ts": 1, "pm7-sparkle": 2, "pm7-minus": 3, "pm7-hh": 4}
ACCELERATORS = {"none": 0, "cdiis": 1, "adiis-cdiis": 2}
REFERENCES = {"auto": 0, "rhf": 1, "uhf": 2}
DIPOLE_ORIGINS = {"coordinates": 0, "centre-of-mass": 1, "centre-of-charge": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}

DP = C.POINTER(C.c_double)


class Molecule(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("z", C.POINTER(C.c_uint8)),
        ("xyz_bohr", DP),
    ]


class EngineConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("method", C.c_int32),
        ("hbm_budget_mb", C.c_int64),
        ("max_active", C.c_int32),
    ]


class Options(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("charge", C.c_double),
        ("multiplicity", C.c_int32),
        ("max_scf", C.c_int32),
        ("e_tol", C.c_double),
        ("p_tol", C.c_double),
        ("use_diis", C.c_int32),
        ("accelerator", C.c_int32),
        ("adiis_switch", C.c_double),
        ("level_shift", C.c_double),
        ("reference", C.c_int32),
        ("force_dpath", C.c_int32),
        ("smooth_dispersion", C.c_int32),
        ("max_memory_mb", C.c_int64),
        ("dipole_origin", C.c_int32),
        ("initial_density", DP),
        ("initial_spin_density", DP),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("want_matrices", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("nao", C.c_int32),
        ("n_occ", C.c_int32),
        ("n_occ_beta", C.c_int32),
        ("unrestricted", C.c_int32),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("density_error", C.c_double),
        ("electronic_ev", C.c_double),
        ("core_ev", C.c_double),
        ("total_ev", C.c_double),
        ("heat_of_formation_kcal", C.c_double),
        ("correction_kcal", C.c_double),
        ("homo_ev", C.c_double),
        ("lumo_ev", C.c_double),
        ("homo_ev_beta", C.c_double),
        ("lumo_ev_beta", C.c_double),
        ("dipole_debye", C.c_double * 3),
        ("dipole_magnitude", C.c_double),
        ("dipole_point_charge", C.c_double * 3),
        ("dipole_sp_hybrid", C.c_double * 3),
        ("dipole_pd_hybrid", C.c_double * 3),
        ("charges", DP),
        ("density", DP),
        ("spin_density", DP),
        ("mo_energies", DP),
        ("mo_coeff", DP),
        ("mo_energies_beta", DP),
        ("mo_coeff_beta", DP),
        ("device_ms", C.c_double),
        ("fp32_iterations", C.c_int32),
    ]


ANGSTROM_TO_BOHR = 1.0 / 0.529177210903  # src/constants.rs:21
EV_TO_HARTREE = 1.0 / 27.211386245988     # src/constants.rs:19


class DandcOptions(C.Structure):
    """`DandcOptions` (pm7-rs src/dandc/mod.rs:62-81)."""
    _fields_ = [
        ("buffer", C.c_double),
        ("core_size", C.c_int32),
        ("fermi_width_ev", C.c_double),
        ("max_scf", C.c_int32),
        ("p_tol", C.c_double),
        ("mixing", C.c_double),
    ]


class DandcResult(C.Structure):
    """`DandcResult` with the energy of `DandcDerivatives` (src/dandc/mod.rs:121-140, 438-443)."""
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("nao", C.c_int32),
        ("converged", C.c_int32),
        ("iterations", C.c_int32),
        ("subsystems", C.c_int32),
        ("largest_subsystem", C.c_int32),
        ("unrestricted", C.c_int32),
        ("fermi_ev", C.c_double),
        ("electronic_ev", C.c_double),
        ("density_error", C.c_double),
        ("core_core_ev", C.c_double),
        ("correction_ev", C.c_double),
        ("energy_ev", C.c_double),
        ("stored_density_elements", C.c_int64),
        ("charges", DP),
        ("gradient", DP),
        ("density", DP),
        ("spin_density", DP),
    ]


def default_dandc_options(**kw):
    """`DandcOptions::default()` (src/dandc/mod.rs:70-81): buffer in Bohr."""
    d = DandcOptions(15.0, 12, 0.1, 200, 1.0e-6, 0.4)
    for k, v in kw.items():
        if not hasattr(d, k):
            raise TypeError(f"unknown divide-and-conquer option {k!r}")
        setattr(d, k, v)
    return d


def default_options(**kw):
    """`Pm7Options::default()` (pm7-rs src/scf.rs:207-233) as an Options struct."""
    o = Options()
    o.method = 0
    o.charge = 0.0
    o.multiplicity = 1
    o.max_scf = 200
    o.e_tol = 1.0e-8
    o.p_tol = 1.0e-7
    o.use_diis = 1
    o.accelerator = 2
    o.adiis_switch = 0.1
    o.level_shift = 0.0
    o.reference = 0
    o.force_dpath = 0
    o.smooth_dispersion = 0
    o.max_memory_mb = -1
    o.dipole_origin = 1
    o.initial_density = None
    o.initial_spin_density = None
    o.precision = 0
    o.device = 0
    o.want_matrices = 1
    for k, v in kw.items():
        if k == "method" and isinstance(v, str):
            v = METHODS[v]
        elif k == "accelerator" and isinstance(v, str):
            v = ACCELERATORS[v]
        elif k == "reference" and isinstance(v, str):
            v = REFERENCES[v]
        elif k == "precision" and isinstance(v, str):
            v = PRECISIONS[v]
        elif k == "dipole_origin" and isinstance(v, str):
            v = DIPOLE_ORIGINS[v]
        setattr(o, k, v)
    return o
