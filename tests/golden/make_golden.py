"""Generate tests/golden/reference_cases.json from the pm7-rs source tree.

Imports pm7-rs tools/oracle/baseline.py (the reference's own case generators:
`CASES`, `COVERAGE` and `OPEN_SHELL`, baseline.py:569,806,960) to regenerate every
case geometry, and pairs each with the pm7-rs results recorded in
tools/oracle/baselines/reference.json (energy, heat of formation, Mulliken charges,
HOMO/LUMO and dipole from the reference CLI at default tolerances,
baseline.py:1086-1113). Run where the pm7-rs tree is available:

    python tests/golden/make_golden.py /path/to/pm7-rs
"""
import json
import sys
from pathlib import Path


def main():
    root = Path(sys.argv[1])
    sys.path.insert(0, str(root / "tools" / "oracle"))
    import baseline  # noqa: E402

    gold = json.loads((root / "tools/oracle/baselines/reference.json").read_text())["cases"]
    out = {}
    for name, (atoms, charge, mult) in baseline.CASES.items():
        rec = gold[name]
        if "pm7_rs" not in rec:  # recorded without a pm7-rs result (thorium_tetrafluoride)
            continue
        out[name] = {
            "atoms": atoms,
            "charge": charge,
            "multiplicity": mult,
            "pm7_rs": rec["pm7_rs"],
        }
    path = Path(__file__).with_name("reference_cases.json")
    path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(out)} cases to {path}")


if __name__ == "__main__":
    main()
