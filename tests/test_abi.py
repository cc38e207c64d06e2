"""The C-ABI library loads and exports every symbol include/pm7_b200.h declares (CPU)."""
import re
from pathlib import Path

import pytest

from pm7b200 import abi, api

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "pm7_b200.h").read_text()
    return sorted(set(re.findall(r"\b(pm7_[a-z_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("pm7_run", "pm7_params_load", "pm7_options_default", "pm7_result_free",
                     "pm7_last_error_message"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = api.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_the_header():
    import ctypes as C

    sizes = api.abi_sizes()
    assert sizes == (C.sizeof(abi.Molecule), C.sizeof(abi.Options), C.sizeof(abi.Result))


def test_dandc_struct_layouts_match_the_header():
    import ctypes as C

    assert api.dandc_abi_sizes() == (C.sizeof(abi.DandcOptions), C.sizeof(abi.DandcResult))


def test_dandc_options_default_matches_reference_defaults():
    import ctypes as C

    d = abi.DandcOptions()
    api.lib().pm7_dandc_options_default(C.byref(d))
    ref = abi.default_dandc_options()
    for name, _ in abi.DandcOptions._fields_:
        assert getattr(d, name) == getattr(ref, name), name
    assert (d.buffer, d.core_size, d.fermi_width_ev, d.max_scf, d.p_tol, d.mixing) == (15.0, 12, 0.1, 200, 1.0e-6, 0.4)


def test_options_default_matches_reference_defaults():
    import ctypes as C

    o = abi.Options()
    api.lib().pm7_options_default(C.byref(o))
    ref = abi.default_options()
    for name, _ in abi.Options._fields_:
        a, b = getattr(o, name), getattr(ref, name)
        if name.startswith("initial"):
            assert not a and not b
        else:
            assert a == b, name


def test_params_load_rejects_unknown_method():
    with pytest.raises(api.Pm7Error) as info:
        api.params(7)
    assert info.value.code == 1


def test_invalid_molecule_is_rejected_before_any_device_work():
    import numpy as np

    with pytest.raises(api.Pm7Error) as info:
        api.run_pm7(np.array([], dtype=np.uint8), np.zeros((0, 3)))
    assert info.value.code == 1
    with pytest.raises(api.Pm7Error) as info:
        api.run_pm7(np.array([1, 1], dtype=np.uint8), np.zeros((2, 3)))
    assert info.value.code == 1
    assert "same position" in api.lib().pm7_last_error_message().decode()


def test_divide_and_conquer_refuses_bad_options_before_any_device_work():
    # option checks (src/dandc/mod.rs:83-110) come before the device is touched
    from pm7b200 import geometry as G

    z, x = G.flat_alkane(2)
    with pytest.raises(api.Pm7Error) as e:
        api.run_dandc(z, x, dandc=dict(buffer=-1.0))
    assert e.value.code == 1 and "buffer" in e.value.message


def test_without_a_device_the_divide_and_conquer_call_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from pm7b200 import geometry as G

    z, x = G.flat_alkane(2)
    with pytest.raises(api.Pm7Error) as e:
        api.run_dandc(z, x)
    assert e.value.code == 9  # PM7_ERR_CUDA: no CPU fallback
