"""XYZ / extended-XYZ input and the JSON output of the reference CLI's `energy --json`.

Wire-format counterparts of pm7-rs `Molecule::from_xyz_str` (src/system.rs:145-197: atom count,
a comment line, then `symbol x y z` in Angstrom; symbols case-insensitive or atomic numbers; a
UTF-8 byte-order mark ignored), `Molecule::to_xyz_string` (:199-231) and the `energy --json`
line of src/bin/pm7_rs.rs:372-441, so scripts that read the reference's files and parse its
JSON can drive this engine unchanged. An extended-XYZ `Lattice=` (a periodic cell) is rejected:
periodic systems are not part of this engine.

    python -m pm7b200.xyz molecule.xyz [--method pm7] [--charge 0] [--multiplicity 1] [--device 0]
"""
import math
import sys

import numpy as np

from . import abi

A0 = 0.529177210903  # Bohr radius in Angstrom (CODATA 2018, src/constants.rs)

# src/system.rs:356-363: index = atomic number
ELEMENTS = [
    "", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S",
    "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
    "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd",
    "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd",
    "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg",
    "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu", "Am", "Cm",
    "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr",
]
_Z_OF = {s: i for i, s in enumerate(ELEMENTS) if s}

METHODS = ["pm7", "pm7-ts", "pm7-sparkle", "pm7-minus", "pm7-hh"]  # src/method.rs:19-27, index = method
_METHOD_ALIASES = {"pm7": 0, "pm7-ts": 1, "pm7ts": 1, "pm7-sparkle": 2, "pm7+sparkle": 2, "sparkle": 2,
                   "pm7-minus": 3, "pm7-": 3, "pm7minus": 3, "pm7-hh": 4, "pm7hh": 4}


class XyzError(ValueError):
    """Malformed or unsupported XYZ input (the reference's `Pm7Error::InvalidInput`, or
    `UnsupportedFeature` for a periodic cell); `.code` is the matching pm7_status."""

    def __init__(self, code, message):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code
        self.message = message


def method_index(name):
    """`Pm7Method::from_str` (src/method.rs:38-52)."""
    key = str(name).strip().lower()
    if key not in _METHOD_ALIASES:
        raise XyzError(1, f"unknown method `{name}`")
    return _METHOD_ALIASES[key]


def symbol_to_z(sym):
    """`symbol_to_z` (src/system.rs:314-327): an atomic number 1..103 or a symbol in any case."""
    try:
        z = int(sym)
        if 1 <= z < len(ELEMENTS):
            return z
    except ValueError:
        pass
    norm = sym[:1].upper() + sym[1:].lower()
    return _Z_OF.get(norm)


def _quoted_value(text, key):
    """The value of `key=...` (quoted or bare) when `key` starts a whitespace-separated word."""
    start = 0
    while True:
        i = text.find(key, start)
        if i < 0:
            return None
        after = text[i + len(key):]
        if (i == 0 or text[i - 1].isspace()) and after.startswith("="):
            after = after[1:]
            if after.startswith('"'):
                return after[1:].split('"', 1)[0]
            return after.split()[0] if after.split() else ""
        start = i + len(key)


def read_xyz(text):
    """Parse an XYZ / extended-XYZ block: returns (z uint8 array, positions in Bohr (N, 3),
    comment line)."""
    if text.startswith("\ufeff"):
        text = text[1:]
    lines = text.splitlines()
    if not lines:
        raise XyzError(1, "empty XYZ")
    try:
        natoms = int(lines[0].strip())
        if natoms < 0:
            raise ValueError
    except ValueError:
        raise XyzError(1, f"invalid XYZ atom count: {lines[0]}") from None
    comment = lines[1] if len(lines) > 1 else ""
    if _quoted_value(comment, "Lattice") is not None:
        raise XyzError(4, "periodic cell (extended-XYZ Lattice): periodic systems are not supported by this engine")
    z, xyz = [], []
    for idx in range(natoms):
        line_no = idx + 3
        if 2 + idx >= len(lines):
            raise XyzError(1, f"XYZ ended before atom {idx}")
        parts = lines[2 + idx].split()
        if len(parts) < 4:
            raise XyzError(1, f"XYZ line {line_no} has fewer than 4 fields")
        zz = symbol_to_z(parts[0])
        if zz is None:
            raise XyzError(1, f"unknown element on line {line_no}: {parts[0]}")
        try:
            pos = [float(parts[1]), float(parts[2]), float(parts[3])]
        except ValueError:
            raise XyzError(1, f"invalid coordinate on line {line_no}") from None
        if not all(math.isfinite(v) for v in pos):
            raise XyzError(1, f"non-finite coordinate on line {line_no}")
        z.append(zz)
        xyz.append([v / A0 for v in pos])
    return np.array(z, dtype=np.uint8), np.array(xyz, dtype=np.float64).reshape(-1, 3), comment


def read_xyz_file(path):
    with open(path, encoding="utf-8") as f:
        return read_xyz(f.read())


def to_xyz_string(z, xyz_bohr, title=""):
    """`Molecule::to_xyz_string` (src/system.rs:199-231), molecular case: Angstrom, 12 decimals."""
    comment = title.replace('"', " ").replace("\n", " ")
    xyz = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    out = [f"{len(xyz)}", comment]
    for zz, p in zip(z, xyz):
        sym = ELEMENTS[int(zz)] if 0 < int(zz) < len(ELEMENTS) else "X"
        out.append(f"{sym} {p[0] * A0:.12f} {p[1] * A0:.12f} {p[2] * A0:.12f}")
    return "\n".join(out) + "\n"


def _f(x):
    return f"{float(x):.12f}"


def _vec(v):
    return "[" + ",".join(_f(x) for x in v) + "]"


def spin_squared(result):
    """`Pm7Result::spin_squared` (src/scf.rs:423-436): S_z(S_z + 1) + n_beta - Tr(P^a P^b), with
    Tr(P^a P^b) = [Tr(P P) - Tr(S S)] / 4; None for RHF or when the densities were not returned."""
    if not result.get("unrestricted") or result.get("density") is None or result.get("spin_density") is None:
        return None
    n_a, n_b = result["n_occ"], result["n_occ_beta"]
    sz = 0.5 * (n_a - n_b)
    p, s = result["density"], result["spin_density"]
    overlap = 0.25 * (float(np.sum(p * p)) - float(np.sum(s * s)))
    return sz * (sz + 1.0) + n_b - overlap


def _present(x):
    return x is not None and math.isfinite(float(x))


def energy_json(result, method="pm7"):
    """The `energy --json` line of the reference CLI (src/bin/pm7_rs.rs:372-441) for a result
    dict of `api.run_pm7`: fields in the same order and 12-decimal format; the optional
    frontier-orbital, gap and <S^2> fields appear when they exist."""
    name = METHODS[method] if isinstance(method, int) else METHODS[method_index(method)]
    fields = [f'"method":"{name}"', f'"energy_ev":{_f(result["total_ev"])}',
              f'"heat_of_formation_kcal":{_f(result["heat_of_formation_kcal"])}',
              '"charges":[' + ",".join(_f(q) for q in result["charges"]) + "]",
              f'"dipole_debye":{_vec(result["dipole_debye"])}',
              f'"dipole_point_charge_debye":{_vec(result["dipole_point_charge"])}',
              f'"dipole_sp_hybrid_debye":{_vec(result["dipole_sp_hybrid"])}',
              f'"dipole_pd_hybrid_debye":{_vec(result["dipole_pd_hybrid"])}',
              '"orbital_source":"molecular"']
    for key in ("homo_ev", "lumo_ev", "homo_ev_beta", "lumo_ev_beta"):
        if _present(result.get(key)):
            fields.append(f'"{key}":{_f(result[key])}')
    homos = [result[k] for k in ("homo_ev", "homo_ev_beta") if _present(result.get(k))]
    lumos = [result[k] for k in ("lumo_ev", "lumo_ev_beta") if _present(result.get(k))]
    if homos and lumos:  # Pm7Result::gap_ev (src/scf.rs:462-473)
        fields.append(f'"gap_ev":{_f(min(lumos) - max(homos))}')
    s2 = spin_squared(result)
    if s2 is not None:
        fields.append(f'"spin_squared":{_f(s2)}')
    return "{" + ",".join(fields) + "}"


def main(argv=None):
    import argparse

    from . import api

    ap = argparse.ArgumentParser(description="PM7 single point of an XYZ file on a B200 (energy --json)")
    ap.add_argument("xyz")
    ap.add_argument("--method", default="pm7")
    ap.add_argument("--charge", type=float, default=0.0)
    ap.add_argument("--multiplicity", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    try:
        z, xyz, _ = read_xyz_file(args.xyz)
        m = method_index(args.method)
        r = api.run_pm7(z, xyz, method=m, charge=args.charge, multiplicity=args.multiplicity, device=args.device,
                        want_matrices=1)
    except (XyzError, api.Pm7Error) as e:
        print(f"error: {e}", file=sys.stderr)
        return 1
    print(energy_json(r, m))
    return 0


if __name__ == "__main__":
    sys.exit(main())
