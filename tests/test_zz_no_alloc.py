"""The allocation-free residual entry point, ostc_compute_residual_noalloc.

It exists for callers that cannot allocate device memory at the time they
want the residual (a host solver that reserves its whole device budget at
start-up, or one sharing a fixed memory pool with other codes); its partial
sums live in a fixed array inside the library. This file is collected last
on purpose: the entry point keeps state on the device between calls, and a
failure here should not hide the results of the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

import ostc

pytestmark = pytest.mark.gpu


def _fn():
    f = ostc.lib().ostc_compute_residual_noalloc
    f.argtypes = [C.POINTER(ostc.Zone), C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_residual_matches_step_residual_on_two_calls():
    import torch

    case = ostc.case_mixing_layer(40, 36, 12, full_host=True)
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    zone = blocks[0].zone()
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):  # the second call finds the first call's partials in the shared array
        res, _dt = s.rk3_steps(1, history=True)  # the existing entry point's residual of this step
        assert _fn()(C.byref(zone), C.c_void_p(out.data_ptr()), stream) == ostc.OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - res[0]) <= 1e-12 * np.abs(res[0])), (got, res[0])
    s.close()


def test_noalloc_rejects_blocks_beyond_its_scratch():
    big = ostc.Zone()
    big.mx, big.my, big.mz, big.ngg = 1024, 1024, 33, 2  # 34.6 M cells > OSTC_NOALLOC_MAX_CELLS
    dummy = (C.c_double * 1)()
    big.bv = big.vel = big.bv_last = C.cast(dummy, C.c_void_p).value
    out = (C.c_double * 4)()
    assert _fn()(C.byref(big), C.cast(out, C.c_void_p), None) == ostc.ERR_INVALID_ARG
