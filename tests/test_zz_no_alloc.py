"""The allocation-free energy entry point, checked against the engine's own.

oems_field_energy_noalloc serves callers that cannot let the library call
cudaMalloc -- a host that owns every byte of device memory and hands the
solver fixed buffers, or a loop that must not stall on the device-wide
synchronisation an allocation can cause.  This test gives it six device
arrays that the test itself allocated (with torch), holding the same fields
as an engine, and compares its energies with oems_engine_energy on two calls
in a row (the second call reuses the library's shared scratch array, so it
also checks that the scratch is reset between calls).  The file is named to
run last, after every other test.
"""
import ctypes

import numpy as np
import pytest

import openems_b200 as oe
from openems_b200 import _native as N

pytestmark = pytest.mark.gpu


def _fields_on_engine(dims, seed):
    op = oe.Operator(oe.Grid.uniform(*dims, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op)
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((6,) + dims).astype(np.float32)
    eng.write_fields(f[:3], f[3:])
    return eng, f


def _noalloc_energy(torch, arrays, stream):
    ptrs = (ctypes.c_void_p * 6)(*[a.data_ptr() for a in arrays])
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    N.check(N.lib().oems_field_energy_noalloc(ptrs, arrays[0].numel(), out.data_ptr(),
                                              ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("dims", [(37, 29, 41), (64, 64, 64)])
def test_noalloc_energy_matches_engine_twice(dims):
    import torch
    stream = torch.cuda.current_stream()
    for call, seed in enumerate((1, 2)):
        eng, f = _fields_on_engine(dims, seed)
        e_ref, h_ref = eng.energy()
        arrays = [torch.from_numpy(np.ascontiguousarray(f[c]).reshape(-1)).cuda() for c in range(6)]
        got = _noalloc_energy(torch, arrays, stream)
        assert got[0] == pytest.approx(e_ref, rel=1e-10), f"call {call + 1}"
        assert got[1] == pytest.approx(h_ref, rel=1e-10), f"call {call + 1}"
        eng.close()


def test_noalloc_rejects_oversized_and_misaligned_input():
    import torch
    a = torch.zeros(8, dtype=torch.float32, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    ptrs = (ctypes.c_void_p * 6)(*([a.data_ptr()] * 6))
    st = N.lib().oems_field_energy_noalloc(ptrs, 67108864 + 1, out.data_ptr(), None)
    assert st == N.ERR_INVALID_ARGUMENT
    assert b"maximum" in N.lib().oems_last_error_message()
    ptrs = (ctypes.c_void_p * 6)(*([a.data_ptr() + 4] * 6))
    assert N.lib().oems_field_energy_noalloc(ptrs, 4, out.data_ptr(), None) == N.ERR_INVALID_ARGUMENT
