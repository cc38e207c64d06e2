"""The device gradient (pm7_gradient) on every recorded reference case against the oracle's
gradient (pinned by tests/test_oracle_gradient.py): sp and MNDO/d frames, transition metals,
lanthanide sparkles, ions and open shells. Each side converges its own SCF, so they agree to
the SCF's convergence: 1e-5 eV/Bohr plus 1e-6 of the component (the recorded geometries are
not relaxed; some forces reach 80 eV/Bohr)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import harness as H
from pm7b200 import api

pytestmark = pytest.mark.gpu

CASES = sorted(json.loads((Path(__file__).resolve().parent / "golden" / "reference_cases.json").read_text()))


@pytest.mark.parametrize("name", CASES)
def test_gradient_golden_case(golden, name):
    case = golden[name]
    z, x = H.parse_lines(case["atoms"])
    opts = dict(charge=float(case["charge"]), multiplicity=case["multiplicity"])
    try:
        _, ref = H.gradient(z, x, **opts)
    except H.OracleError as e:
        with pytest.raises(api.Pm7Error) as info:
            api.closed_form_gradient(z, x, **opts)
        assert info.value.code == e.code
        return
    out = api.closed_form_gradient(z, x, **opts)
    diff = np.abs(out["gradient"] - ref)
    assert np.all(diff <= 1.0e-5 + 1.0e-6 * np.abs(ref)), (name, float(diff.max()), float(np.abs(ref).max()))
