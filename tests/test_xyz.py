"""XYZ input and the `energy --json` output shape (CPU).

The reference reads molecules from XYZ files (src/system.rs:145-197) and its oracle scripts read
results from `pm7_rs energy --json` (src/bin/pm7_rs.rs:372-441). `pm7b200.xyz` mirrors both.
The recorded reference results in tests/golden/reference_cases.json are that JSON: formatting
the oracle's result for the same molecule must give the same keys (including the optional
beta-orbital, gap and <S^2> fields) and the same values.
"""
import json

import numpy as np
import pytest

from oracle import harness
from pm7b200 import xyz as X

WATER = "3\nwater\nO 0.0 0.0 0.0\nH 0.96 0.0 0.0\nH -0.24 0.93 0.0\n"


def test_read_xyz_basic_and_units():
    z, x, comment = X.read_xyz(WATER)
    assert list(z) == [8, 1, 1] and comment == "water"
    assert x[1, 0] == pytest.approx(0.96 / 0.529177210903, rel=1e-15)


def test_read_xyz_symbols_numbers_bom_and_extra_columns():
    text = "\ufeff3\n\no 0 0 0 extra\n1 0.96 0 0\nh -0.24 0.93 0 1.0\n"
    z, x, _ = X.read_xyz(text)
    assert list(z) == [8, 1, 1]
    assert X.symbol_to_z("CL") == 17 and X.symbol_to_z("103") == 103 and X.symbol_to_z("104") is None


@pytest.mark.parametrize("text,code,what", [
    ("", 1, "empty"), ("x\n\n", 1, "atom count"), ("2\n\nO 0 0 0\n", 1, "ended before atom 1"),
    ("1\n\nO 0 0\n", 1, "fewer than 4 fields"), ("1\n\nQq 0 0 0\n", 1, "unknown element"),
    ("1\n\nO 0 zero 0\n", 1, "invalid coordinate"),
    ('1\nLattice="5 0 0 0 5 0 0 0 5" pbc="T T T"\nO 0 0 0\n', 4, "periodic"),
])
def test_read_xyz_errors(text, code, what):
    with pytest.raises(X.XyzError) as info:
        X.read_xyz(text)
    assert info.value.code == code and what in info.value.message


def test_xyz_round_trip():
    z, x, _ = X.read_xyz(WATER)
    z2, x2, c2 = X.read_xyz(X.to_xyz_string(z, x, 'a "title"'))
    assert list(z2) == list(z) and np.max(np.abs(x2 - x)) < 1e-12 and c2 == "a  title "


def test_method_names():
    assert [X.method_index(m) for m in ("PM7", "pm7-ts", "sparkle", "pm7-", "PM7HH")] == [0, 1, 2, 3, 4]
    with pytest.raises(X.XyzError):
        X.method_index("am1")


def _cases(golden):
    names = sorted(golden)
    pick = names[:12] + [n for n in names if golden[n]["multiplicity"] > 1]
    pick += [n for n in names if "lumo_ev" not in golden[n]["pm7_rs"]]
    return sorted(set(pick))


def test_energy_json_matches_recorded_reference_output(golden):
    for name in _cases(golden):
        case = golden[name]
        z, x = harness.parse_lines(case["atoms"])
        r = harness.run(z, x, charge=float(case["charge"]), multiplicity=case["multiplicity"], want_matrices=1)
        line = X.energy_json(r, "pm7")
        out = json.loads(line)
        ref = case["pm7_rs"]
        assert set(out) == set(ref), (name, set(out) ^ set(ref))
        for k, v in ref.items():
            if isinstance(v, str):
                assert out[k] == v, (name, k)
            else:
                assert np.allclose(out[k], v, rtol=0, atol=1e-6), (name, k, out[k], v)
