"""Python harness of the CPU oracle (test infrastructure only).

Loads oracle/_build/libpm7oracle.so — the C++ restatement of pm7-rs `run_pm7` — and
exposes it with the same argument meaning as the engine's public API so parity tests
read like the reference's own tests. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import glob
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "pm7-rs_b200"))
from pm7b200 import abi  # noqa: E402

LIB_PATH = ROOT / "oracle" / "_build" / "libpm7oracle.so"

SYMBOLS = [
    "X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar",
    "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe",
    "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf",
    "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U", "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No",
]
Z_OF = {s: i for i, s in enumerate(SYMBOLS)}
A0 = 0.529177210903

_lib = None


class OracleError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} not built; run `make -C oracle`")
    L = C.CDLL(str(LIB_PATH))
    L.pm7_oracle_set_lapack.argtypes = [C.c_char_p, C.c_int]
    L.pm7_oracle_set_lapack.restype = C.c_int
    L.pm7_oracle_set_threads.argtypes = [C.c_int]
    L.pm7_oracle_last_error.restype = C.c_char_p
    L.pm7_oracle_run.argtypes = [C.POINTER(abi.Molecule), C.POINTER(abi.Options), C.POINTER(abi.Result)]
    L.pm7_oracle_result_free.argtypes = [C.POINTER(abi.Result)]
    L.pm7_oracle_core_hamiltonian.argtypes = [C.POINTER(abi.Molecule), C.c_int, C.c_int, abi.DP, C.POINTER(C.c_int)]
    L.pm7_oracle_fock.argtypes = [C.POINTER(abi.Molecule), C.c_int, C.c_int, abi.DP, abi.DP, abi.DP]
    L.pm7_oracle_pair.argtypes = [C.c_int, C.c_int, C.c_int, abi.DP, C.c_int, abi.DP, abi.DP, abi.DP, abi.DP,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pm7_oracle_core_core.argtypes = [C.POINTER(abi.Molecule), C.c_int, abi.DP]
    L.pm7_oracle_corrections.argtypes = [C.POINTER(abi.Molecule), C.c_int, C.c_int, abi.DP]
    L.pm7_oracle_element.argtypes = [C.c_int, C.c_int, abi.DP]
    L.pm7_oracle_fixed_density_gradient.argtypes = [C.POINTER(abi.Molecule), C.c_int, C.c_int, abi.DP, abi.DP,
                                                    C.c_double, abi.DP]
    L.pm7_oracle_run_dandc.argtypes = [C.POINTER(abi.Molecule), C.POINTER(abi.Options), C.POINTER(abi.DandcOptions),
                                       C.POINTER(abi.DandcResult)]
    L.pm7_oracle_dandc_result_free.argtypes = [C.POINTER(abi.DandcResult)]
    L.pm7_oracle_dandc_partition.argtypes = [C.POINTER(abi.Molecule), C.c_int32, C.c_double, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.pm7_oracle_correction_gradient.argtypes = [C.POINTER(abi.Molecule), C.c_int, C.c_int, C.c_double, abi.DP]
    libs = sorted(glob.glob(os.path.join(os.path.dirname(np.__file__) + ".libs", "libscipy_openblas64_*.so")))
    if libs:
        L.pm7_oracle_set_lapack(libs[0].encode(), int(os.environ.get("PM7_ORACLE_BLAS_THREADS", "0")))
    _lib = L
    return L


def set_threads(n):
    lib().pm7_oracle_set_threads(int(n))


def parse_lines(lines):
    """`"El x y z"` lines in Angstrom -> (Z uint8 array, positions in Bohr (N,3))."""
    z, xyz = [], []
    for line in lines:
        parts = line.split()
        z.append(Z_OF[parts[0]])
        xyz.append([float(parts[1]) / A0, float(parts[2]) / A0, float(parts[3]) / A0])
    return np.array(z, dtype=np.uint8), np.array(xyz, dtype=np.float64).reshape(-1, 3)


class _Mol:
    def __init__(self, z, xyz_bohr):
        self.z = np.ascontiguousarray(z, dtype=np.uint8)
        self.xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1)
        self.s = abi.Molecule(len(self.z), self.z.ctypes.data_as(C.POINTER(C.c_uint8)),
                              self.xyz.ctypes.data_as(abi.DP))


def _check(code):
    if code != 0:
        raise OracleError(code, lib().pm7_oracle_last_error().decode())


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


def run(z, xyz_bohr, **options):
    """Oracle `run_pm7`: returns a dict of the result fields; raises OracleError."""
    m = _Mol(z, xyz_bohr)
    keep = []
    for k in ("initial_density", "initial_spin_density"):
        if options.get(k) is not None:
            a = np.ascontiguousarray(options[k], dtype=np.float64)
            keep.append(a)
            options[k] = a.ctypes.data_as(abi.DP)
    o = abi.default_options(**options)
    r = abi.Result()
    code = lib().pm7_oracle_run(C.byref(m.s), C.byref(o), C.byref(r))
    if code != 0:
        raise OracleError(code, lib().pm7_oracle_last_error().decode())
    try:
        return result_to_dict(r)
    finally:
        lib().pm7_oracle_result_free(C.byref(r))


def sample(z, xyz_bohr, n_iter, **options):
    """Timed bounded sample: (build s, seconds of n_iter iterations, post-SCF s, iterations)."""
    L = lib()
    L.pm7_oracle_sample.argtypes = [C.POINTER(abi.Molecule), C.POINTER(abi.Options), C.c_int, abi.DP]
    m = _Mol(z, xyz_bohr)
    o = abi.default_options(**options)
    out = np.zeros(4)
    _check(L.pm7_oracle_sample(C.byref(m.s), C.byref(o), int(n_iter), out.ctypes.data_as(abi.DP)))
    return tuple(out)


def core_hamiltonian(z, xyz_bohr, method=0, force_dpath=False):
    m = _Mol(z, xyz_bohr)
    nao = C.c_int()
    _check(lib().pm7_oracle_core_hamiltonian(C.byref(m.s), method, int(force_dpath), None, C.byref(nao)))
    h = np.zeros((nao.value, nao.value))
    _check(lib().pm7_oracle_core_hamiltonian(C.byref(m.s), method, int(force_dpath), h.ctypes.data_as(abi.DP),
                                             C.byref(nao)))
    return h


def fock(z, xyz_bohr, p_tot, p_spin, method=0, force_dpath=False):
    m = _Mol(z, xyz_bohr)
    pt = np.ascontiguousarray(p_tot, dtype=np.float64)
    ps = np.ascontiguousarray(p_spin, dtype=np.float64)
    f = np.zeros_like(pt)
    _check(lib().pm7_oracle_fock(C.byref(m.s), method, int(force_dpath), pt.ctypes.data_as(abi.DP),
                                 ps.ctypes.data_as(abi.DP), f.ctypes.data_as(abi.DP)))
    return f


def pair(zi, zj, d, method=0, force_dpath=False):
    dd = np.ascontiguousarray(d, dtype=np.float64)
    w = np.zeros(45 * 45)
    e1b, e2a, s = np.zeros(81), np.zeros(81), np.zeros(81)
    npi, npj = C.c_int(), C.c_int()
    _check(lib().pm7_oracle_pair(method, zi, zj, dd.ctypes.data_as(abi.DP), int(force_dpath),
                                 w.ctypes.data_as(abi.DP), e1b.ctypes.data_as(abi.DP), e2a.ctypes.data_as(abi.DP),
                                 s.ctypes.data_as(abi.DP), C.byref(npi), C.byref(npj)))
    return (w[: npi.value * npj.value].reshape(npi.value, npj.value), e1b.reshape(9, 9), e2a.reshape(9, 9),
            s.reshape(9, 9))


def core_core(z, xyz_bohr, method=0):
    m = _Mol(z, xyz_bohr)
    e = C.c_double()
    _check(lib().pm7_oracle_core_core(C.byref(m.s), method, C.byref(e)))
    return e.value


def corrections(z, xyz_bohr, method=0, smooth=False):
    m = _Mol(z, xyz_bohr)
    out = np.zeros(5)
    _check(lib().pm7_oracle_corrections(C.byref(m.s), method, int(smooth), out.ctypes.data_as(abi.DP)))
    return out


def fixed_density_gradient(z, xyz_bohr, p_total, p_spin=None, method=0, force_dpath=False, step=1.0e-3):
    """Core-core + electronic gradient (eV/Bohr) at a fixed density: the five-point difference
    of `energy_at_fixed_density_with` (src/gradient.rs:312-432)."""
    m = _Mol(z, xyz_bohr)
    pt = np.ascontiguousarray(p_total, dtype=np.float64)
    ps = None if p_spin is None else np.ascontiguousarray(p_spin, dtype=np.float64)
    g = np.zeros((len(m.z), 3))
    _check(lib().pm7_oracle_fixed_density_gradient(C.byref(m.s), method, int(force_dpath), pt.ctypes.data_as(abi.DP),
                                                   None if ps is None else ps.ctypes.data_as(abi.DP), step,
                                                   g.ctypes.data_as(abi.DP)))
    return g


def correction_gradient(z, xyz_bohr, method=0, smooth=False, step=1.0e-5):
    """Post-SCF correction gradient (eV/Bohr, src/gradient.rs:208-261) by the five-point
    difference of the correction energy. The step is small because the EH+ H-bond energy
    has kinks (hard switches); a wider stencil can straddle one."""
    m = _Mol(z, xyz_bohr)
    g = np.zeros((len(m.z), 3))
    _check(lib().pm7_oracle_correction_gradient(C.byref(m.s), method, int(smooth), step, g.ctypes.data_as(abi.DP)))
    return g


def gradient(z, xyz_bohr, step=1.0e-3, corr_step=1.0e-5, **options):
    """The closed-form gradient's quantities (src/gradient.rs:500-561) from the oracle: its
    SCF, then the fixed-density and correction gradients at the converged density."""
    r = run(z, xyz_bohr, want_matrices=1, **options)
    method = options.get("method", 0)
    g = fixed_density_gradient(z, xyz_bohr, r["density"], r["spin_density"] if r["unrestricted"] else None,
                               method=method, force_dpath=options.get("force_dpath", False), step=step)
    g = g + correction_gradient(z, xyz_bohr, method=method, smooth=options.get("smooth_dispersion", False),
                                step=corr_step)
    return r, g


def dandc_partition(z, xyz_bohr, core_size=12, buffer=15.0):
    """The oracle's divide-and-conquer partition (src/dandc/partition.rs): (core_of, sizes,
    stored atom pairs), in the layout of the engine's pm7_stage_dandc_partition."""
    m = _Mol(z, xyz_bohr)
    n = len(m.z)
    core_of = np.zeros(n, dtype=np.int32)
    sizes = np.zeros(max(n, 1), dtype=np.int32)
    count = C.c_int32()
    pairs = C.c_int64()
    _check(lib().pm7_oracle_dandc_partition(C.byref(m.s), int(core_size), float(buffer),
                                            core_of.ctypes.data_as(C.POINTER(C.c_int32)),
                                            sizes.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(count),
                                            C.byref(pairs)))
    return core_of, sizes[:count.value].copy(), pairs.value


def run_dandc(z, xyz_bohr, dandc=None, gradient=False, step=1.0e-3, corr_step=1.0e-5, **options):
    """Oracle `run_dandc` (src/dandc/mod.rs:143-428): the result fields as a dict (the dense
    global density under want_matrices). With `gradient`, `dandc_derivatives`' gradient
    (:462-481): the RHF fixed-density gradient of the total density plus the correction
    gradient."""
    m = _Mol(z, xyz_bohr)
    want = gradient or options.get("want_matrices", 1)
    options = dict(options, want_matrices=int(bool(want)))
    o = abi.default_options(**options)
    d = abi.default_dandc_options(**(dandc or {}))
    r = abi.DandcResult()
    code = lib().pm7_oracle_run_dandc(C.byref(m.s), C.byref(o), C.byref(d), C.byref(r))
    if code != 0:
        raise OracleError(code, lib().pm7_oracle_last_error().decode())
    try:
        n, nao = r.n_atoms, r.nao
        out = {k: getattr(r, k) for k in ("n_atoms", "nao", "converged", "iterations", "subsystems",
                                           "largest_subsystem", "unrestricted", "fermi_ev", "electronic_ev",
                                           "density_error", "core_core_ev", "correction_ev", "energy_ev",
                                           "stored_density_elements")}
        out["converged"] = bool(out["converged"])
        out["unrestricted"] = bool(out["unrestricted"])
        out["charges"] = _arr(r.charges, n)
        for k in ("density", "spin_density"):
            a = _arr(getattr(r, k), nao * nao)
            out[k] = None if a is None else a.reshape(nao, nao)
    finally:
        lib().pm7_oracle_dandc_result_free(C.byref(r))
    if gradient:
        method = options.get("method", 0)
        g = fixed_density_gradient(z, xyz_bohr, out["density"], None, method=method, step=step)
        out["gradient"] = g + correction_gradient(z, xyz_bohr, method=method,
                                                  smooth=options.get("smooth_dispersion", False), step=corr_step)
    return out


def numerical_gradient(z, xyz_bohr, step=1.0e-4, **options):
    """`numerical_gradient` (src/gradient.rs:454-498): central difference of the full SCF's
    total energy."""
    x0 = np.array(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    g = np.zeros_like(x0)
    for a in range(len(x0)):
        for k in range(3):
            e = []
            for t in (step, -step):
                x = x0.copy()
                x[a, k] += t
                e.append(run(z, x, want_matrices=0, **options)["total_ev"])
            g[a, k] = (e[0] - e[1]) / (2.0 * step)
    return g


def element(z, method=0):
    out = np.zeros(24)
    _check(lib().pm7_oracle_element(method, z, out.ctypes.data_as(abi.DP)))
    return out
