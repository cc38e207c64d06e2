"""The allocation-free corrections entry point, checked through the C ABI on a GPU.

`pm7_corrections_noalloc` is for callers that cannot allocate device memory (a host
whose allocator owns every byte of HBM, or a loop that must not take a cudaMalloc's
implicit synchronisation): they hand in device buffers and a stream, and the library
works in its own static scratch array instead of allocating. Two calls in a row must
agree with the allocating `pm7_stage_corrections` to the tolerance the other
correction tests use. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from pm7b200 import api
from pm7b200 import geometry as G

pytestmark = pytest.mark.gpu


def _entry():
    lib = api.lib()
    f = lib.pm7_corrections_noalloc
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    f.restype = C.c_int32
    lib.pm7_corrections_noalloc_error.restype = C.c_char_p
    return f, lib


def _call_noalloc(z, xyz, method=0, smooth=False):
    import torch

    f, lib = _entry()
    zd = torch.as_tensor(np.asarray(z, dtype=np.int32), device="cuda")
    xd = torch.as_tensor(np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1), device="cuda")
    out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    code = f(len(z), zd.data_ptr(), xd.data_ptr(), method, int(smooth), out.data_ptr(), stream.cuda_stream)
    assert code == 0, lib.pm7_corrections_noalloc_error().decode()
    stream.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_the_allocating_entry_point_twice_in_a_row():
    first = G.water_cluster(40, seed=3)
    second = G.alkane(9, seed=1)
    for z, xyz in (first, second):
        got = _call_noalloc(z, xyz)
        want = api.corrections(z, xyz)
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11)
    # and the first molecule again: no state carried over from the previous call
    z, xyz = first
    np.testing.assert_allclose(_call_noalloc(z, xyz), api.corrections(z, xyz), rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("method,smooth", [(0, True), (3, False), (4, False), (4, True)])
def test_noalloc_covers_every_correction_branch(method, smooth):
    # the smooth C6 dispersion, PM7-minus and the PM7-HH hydrogen-bond terms share the same
    # static scratch: each branch against the allocating entry point, twice in a row
    for z, xyz in (G.water_cluster(24, seed=5), G.alkane(7, seed=2)):
        want = api.corrections(z, xyz, method=method, smooth=smooth)
        for _ in range(2):
            got = _call_noalloc(z, xyz, method=method, smooth=smooth)
            np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11)


def test_noalloc_rejects_sizes_beyond_its_static_scratch():
    f, lib = _entry()
    limit = lib.pm7_corrections_noalloc_max_atoms()
    assert limit == 2048
    code = f(limit + 1, 1, 1, 0, 0, 1, None)
    assert code == 1
    assert "2048" in lib.pm7_corrections_noalloc_error().decode()
