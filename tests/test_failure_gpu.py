"""Failure detection of the path, made on the host and never by a GPU fault:

* a NaN planted in a host-prepared input is reported as OSTC_ERR_NONPHYSICAL
  with its block and cell by the residual epilogue's state check (the
  reference stops on a NaN residual, src/Residual.cuh:153-158), on the RK3
  and the steady drivers, and the context keeps working once the caller
  restores a valid state;
* a bounded tensor-core wait that runs out (its completion signal withheld
  on request, a flag that nothing sets) is reported as OSTC_ERR_TIMEOUT after
  about a second, and the next call gives the normal result;
* likewise the bounded grid barrier between the waves of the batched
  boundary-face and interface launches (its release withheld on request):
  the steps with histories return OSTC_ERR_TIMEOUT and, with the release
  restored, the same context steps as a fresh one.
"""
import time

import numpy as np
import pytest

import ostc

pytestmark = pytest.mark.gpu


def _plant_nan(case, cell, plane=0):
    b = case.blocks[0]
    g = b.ngg
    i, j, k = cell
    b.arrays["bv"][plane, k + g, j + g, i + g] = np.nan


def _reach_ok(err, cell, reach):
    st, _cuda, blk, i, j, k = err
    return st == ostc.ERR_NONPHYSICAL and blk == 0 and all(abs(a - b) <= reach for a, b in zip((i, j, k), cell))


def test_nan_in_input_reported_by_rk3_steps():
    cell = (12, 9, 4)
    clean = ostc.case_vortex(32, 24, 8)
    case = ostc.case_vortex(32, 24, 8)
    _plant_nan(case, cell)
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    with pytest.raises(ostc.OstcError) as e:
        s.rk3_steps(2, history=True)
    assert e.value.status == ostc.ERR_NONPHYSICAL
    err = s.get_error()
    # the NaN spreads by the stencil (3 cells per stage at most) before the
    # first check at the end of step 1
    assert _reach_ok(err, cell, 9), err
    # the caller restores a valid state: the same context steps cleanly
    blocks[0].upload("bv", clean.blocks[0].arrays["bv"])
    s.initialize()
    res, _ = s.rk3_steps(2, history=True)
    assert np.all(np.isfinite(res)) and np.all(res > 0)
    s.close()


def test_nan_in_input_reported_by_steady_steps():
    case = ostc.make_steady(ostc.case_premixed_box(16, 14, 8), implicit_method=1)
    cell = (7, 6, 3)
    _plant_nan(case, cell, plane=5)  # temperature
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    with pytest.raises(ostc.OstcError) as e:
        s.steady_steps(2, history=True)
    assert e.value.status == ostc.ERR_NONPHYSICAL
    assert _reach_ok(s.get_error(), cell, 8), s.get_error()
    s.close()


def test_bounded_tensor_core_wait_runs_out_and_recovers():
    import torch

    sur = ostc.Surrogate(max_batch=4096, seed=3)
    xs = torch.randn(1000, ostc.SURR_IN, device="cuda", dtype=torch.float32)
    y_ref = sur.forward_tc(xs).clone()
    sur.inject_timeout(True)
    t0 = time.perf_counter()
    with pytest.raises(ostc.OstcError) as e:
        sur.forward_tc(xs)
    waited = time.perf_counter() - t0
    assert e.value.status == ostc.ERR_TIMEOUT
    assert 0.5 < waited < 10.0, waited
    sur.inject_timeout(False)
    y = sur.forward_tc(xs)
    torch.cuda.synchronize()
    assert torch.equal(y, y_ref)
    sur.close()


def test_bounded_wave_barrier_runs_out_and_recovers():
    def make():
        return ostc.case_uneven_blocks(
            layout=ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False),
            rans_model=2)

    ref_case = make()
    s_ref, _ = ref_case.solver()
    s_ref.initialize()
    res_ref, dt_ref = s_ref.rk3_steps(2, history=True)
    s_ref.close()

    s, blocks = make().solver()
    assert s.batching()
    s.initialize()
    s.inject_wave_timeout(True)
    t0 = time.perf_counter()
    with pytest.raises(ostc.OstcError) as e:
        s.rk3_steps(1, history=True)
    waited = time.perf_counter() - t0
    assert e.value.status == ostc.ERR_TIMEOUT
    assert 0.5 < waited < 60.0, waited
    s.inject_wave_timeout(False)
    # the state after the withheld waves is not valid: start again from the inputs
    for b, h in zip(blocks, make().blocks):
        b.upload_inputs(h)
    s.initialize()
    res, dts = s.rk3_steps(2, history=True)
    assert np.array_equal(res, res_ref) and np.array_equal(dts, dt_ref)
    s.close()
