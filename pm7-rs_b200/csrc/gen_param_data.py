"""Generate pm7_param_data.h: the PM7 parameter tables as C arrays.

The tables are data, not code: MOPAC v23.2.5 PM7 / PM7-TS element, pair and
global-correction parameters (Apache-2.0, (c) 2021 Virginia Tech), as
distributed in CSV form by pm7-rs (src/data/*.csv), plus the MNDO/d index and
multipole-coefficient tables (pm7-rs src/mndod_tables.rs, generated there from
MOPAC src/integrals/mndod.F90) and the atomic-mass table (pm7-rs
src/data_tables.rs:19). Run once with the pm7-rs source tree available:

    python gen_param_data.py /path/to/pm7-rs > pm7_param_data.h

Every number is copied verbatim as text so the C parser reads the same double
the reference's Rust parser reads.
"""
import re
import sys
from pathlib import Path

ELEMENT_COLUMNS = [
    "z", "n", "ios", "iop", "iod", "core_charge", "eheat_kcal", "u_ss", "u_pp", "u_dd",
    "zeta_s", "zeta_p", "zeta_d", "beta_s", "beta_p", "beta_d", "g_ss", "g_sp", "g_pp",
    "g_p2", "h_sp", "zsn", "zpn", "zdn", "f0sd", "g2sd", "alpha", "poc", "polvol",
    "g1_1", "g1_2", "g1_3", "g1_4", "g2_1", "g2_2", "g2_3", "g2_4", "g3_1", "g3_2",
    "g3_3", "g3_4",
]


def csv_rows(path):
    lines = [l.strip() for l in Path(path).read_text().splitlines()]
    lines = [l for l in lines if l and not l.startswith("#")]
    header = [h.strip() for h in lines[0].split(",")]
    return header, [[f.strip() for f in l.split(",")] for l in lines[1:]]


def emit_elements(name, path):
    header, rows = csv_rows(path)
    idx = [header.index(c) for c in ELEMENT_COLUMNS]
    out = [f"static const double {name}[][{len(ELEMENT_COLUMNS)}] = {{"]
    for r in rows:
        out.append("  {" + ", ".join(r[i] for i in idx) + "},")
    out.append("};")
    out.append(f"static const int {name}_ROWS = {len(rows)};")
    return "\n".join(out)


def emit_pairs(name, path):
    header, rows = csv_rows(path)
    idx = [header.index(c) for c in ("z_hi", "z_lo", "alpb", "xfac")]
    out = [f"static const double {name}[][4] = {{"]
    for r in rows:
        out.append("  {" + ", ".join(r[i] for i in idx) + "},")
    out.append("};")
    out.append(f"static const int {name}_ROWS = {len(rows)};")
    return "\n".join(out)


def emit_vpar(name, path):
    header, rows = csv_rows(path)
    i, v = header.index("index"), header.index("value")
    out = [f"static const double {name}[][2] = {{"]
    for r in rows:
        out.append(f"  {{{r[i]}, {r[v]}}},")
    out.append("};")
    out.append(f"static const int {name}_ROWS = {len(rows)};")
    return "\n".join(out)


def emit_sparkles(name, path):
    header, rows = csv_rows(path)
    cols = ["z", "alpha", "g_ss", "g1_1", "g2_1", "g3_1", "g1_2", "g2_2", "g3_2"]
    idx = [header.index(c) for c in cols]
    out = [f"/* columns: {' '.join(cols)} */", f"static const double {name}[][{len(cols)}] = {{"]
    for r in rows:
        out.append("  {" + ", ".join(r[i] for i in idx) + "},")
    out.append("};")
    out.append(f"static const int {name}_ROWS = {len(rows)};")
    return "\n".join(out)


def rust_array(text, name):
    m = re.search(rf"pub (?:static|const) {name}: \[(\w+); (\d+)\] = \[(.*?)\];", text, re.S)
    if not m:
        raise SystemExit(f"array {name} not found")
    ty, n, body = m.group(1), int(m.group(2)), m.group(3)
    vals = [v.strip() for v in body.replace("\n", " ").split(",") if v.strip()]
    if len(vals) != n:
        raise SystemExit(f"{name}: expected {n} values, got {len(vals)}")
    return ty, vals


CTYPE = {"u16": "unsigned short", "i16": "short", "u8": "unsigned char", "f64": "double"}


def emit_rust(text, name, cname):
    ty, vals = rust_array(text, name)
    lines = [f"static const {CTYPE[ty]} {cname}[{len(vals)}] = {{"]
    for k in range(0, len(vals), 12):
        lines.append("  " + ", ".join(vals[k:k + 12]) + ",")
    lines.append("};")
    return "\n".join(lines)


def main():
    root = Path(sys.argv[1])
    data = root / "src/data"
    tables = (root / "src/mndod_tables.rs").read_text()
    dt = (root / "src/data_tables.rs").read_text()
    parts = [
        "/* Generated by gen_param_data.py; do not edit by hand. */",
        "/* PM7 / PM7-TS parameters: MOPAC v23.2.5 (Apache-2.0, (c) 2021 Virginia Tech). */",
        "#pragma once",
        f"/* element columns: {' '.join(ELEMENT_COLUMNS)} */",
        f"#define PM7_ELEMENT_NCOL {len(ELEMENT_COLUMNS)}",
        emit_elements("PM7_ELEMENTS", data / "pm7_elements.csv"),
        emit_pairs("PM7_PAIRS", data / "pm7_pairs.csv"),
        emit_vpar("PM7_VPAR", data / "pm7_vpar.csv"),
        emit_elements("PM7TS_ELEMENTS", data / "pm7ts_elements.csv"),
        emit_pairs("PM7TS_PAIRS", data / "pm7ts_pairs.csv"),
        emit_vpar("PM7TS_VPAR", data / "pm7ts_vpar.csv"),
        emit_sparkles("PM7_SPARKLES", data / "pm7_sparkles.csv"),
        "/* MNDO/d tables (MOPAC mndod.F90 fordd), 1-based values as in MOPAC. */",
        emit_rust(tables, "IND2", "MNDOD_IND2"),
        emit_rust(tables, "ISYM", "MNDOD_ISYM"),
        emit_rust(tables, "CH", "MNDOD_CH"),
        emit_rust(tables, "INDPP", "MNDOD_INDPP"),
        emit_rust(tables, "INDDP", "MNDOD_INDDP"),
        emit_rust(tables, "INDDD", "MNDOD_INDDD"),
        emit_rust(tables, "INTIJ", "MNDOD_INTIJ"),
        emit_rust(tables, "INTKL", "MNDOD_INTKL"),
        emit_rust(tables, "INTREP", "MNDOD_INTREP"),
        "/* Atomic masses (u) by Z, 0 = none. */",
        emit_rust(dt, "MASS", "PM7_MASS"),
    ]
    print("\n\n".join(parts))


if __name__ == "__main__":
    main()
