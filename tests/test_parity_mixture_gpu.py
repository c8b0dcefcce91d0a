"""GPU parity of the 9-species H2-air path (MUSCL/NND2/first-order
reconstruction + AUSM+/HLLC, mixture thermodynamics and transport,
finite-rate chemistry source, Newton temperature solve) against the CPU
oracle, through the C ABI.

Tolerances as for air: 1e-11 per RHS evaluation in the conditioning-aware
normwise measure of tests/oracle_bind.py (rhs_errors); properties 1e-12
relative; 1e-9 on multi-step histories.
"""
import numpy as np
import pytest

import ostc
from oracle_bind import OracleRun, normwise, rhs_errors

pytestmark = pytest.mark.gpu
RHS_TOL = 1e-11


def _case(shape, **kw):
    return ostc.case_mixing_layer(*shape, full_host=True, **kw)


def _gpu(case):
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    return ostc.Solver(case.scheme, case.mech, blocks, case.faces), blocks


def test_properties_match():
    case = _case((24, 20, 8))
    ref = OracleRun(case)
    ref.initialize()
    s, blocks = _gpu(case)
    s.initialize()
    hb = ref.blocks[0].arrays
    for name in ("cv", "mul", "thermal_conductivity", "rho_D", "gamma", "cp", "acoustic_speed"):
        got = blocks[0].download(name)
        den = np.max(np.abs(hb[name]))
        assert np.max(np.abs(got - hb[name])) <= 1e-12 * den, name


@pytest.mark.parametrize("rec,flux", [(2, 3), (3, 3), (1, 3), (2, 4), (3, 4), (2, 2), (1, 2)])
@pytest.mark.parametrize("shape", [(24, 20, 8), (33, 17, 10)])
def test_rhs_matches_oracle(shape, rec, flux):
    case = _case(shape)
    case.scheme.reconstruction = rec
    case.scheme.inviscid_scheme = flux
    ref = OracleRun(case)
    ref.initialize()
    scale = ref.flux_scale()
    s, blocks = _gpu(case)
    s.initialize()
    s.compute_rhs()
    err = rhs_errors(blocks[0].download("dq"), ref.blocks[0].arrays["dq"], scale)
    assert max(err) <= RHS_TOL, err


def test_rk3_history_matches_oracle():
    case = _case((24, 20, 8))
    n = 6
    ref = OracleRun(case)
    ref.initialize()
    res_o, dt_o = ref.rk3_steps(n)
    s, blocks = _gpu(case)
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for name in ("bv", "sv"):
        err = normwise(blocks[0].download(name), ref.blocks[0].arrays[name])
        assert max(err) <= 1e-9, (name, err)


def test_inviscid_only_and_no_reactions():
    case = _case((20, 16, 8))
    case.scheme.viscous_order = 0
    ref = OracleRun(case)
    ref.initialize()
    scale = ref.flux_scale()
    s, blocks = _gpu(case)
    s.initialize()
    s.compute_rhs()
    assert max(rhs_errors(blocks[0].download("dq"), ref.blocks[0].arrays["dq"], scale)) <= RHS_TOL


def test_generated_chemistry_matches_generic():
    """The generated straight-line chemistry (mech_h2air9.cuh) against the
    generic loops on the same RHS: the same operations up to FMA
    contraction, so agreement to 1e-13 of the flux scale."""
    from oracle_bind import OracleRun, rhs_errors

    case = ostc.case_premixed_box(16, 14, 8, dx=1e-3, T0=1500.0)
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale()
    out = []
    for gen in (True, False):
        s, blocks = case.solver()
        s.use_generated_chemistry(gen)
        s.initialize()
        s.compute_rhs()
        out.append(blocks[0].download("dq"))
        s.close()
    assert max(rhs_errors(out[0], out[1], scale)) <= 1e-13
    assert max(rhs_errors(out[0], o.blocks[0].arrays["dq"], scale)) <= 1e-11


@pytest.mark.parametrize("rec,flux", [(2, 3), (3, 4), (2, 2)])
@pytest.mark.parametrize("vtile", [((4 | 2 << 8), 3), ((8 | 3 << 8), 1), ((2 | 4 << 8), 2)])
def test_split_flux_matches_oracle(rec, flux, vtile):
    """Inviscid and viscous fluxes as two kernels per direction (tile of
    directions 3..5 set) against the oracle, and against the fused kernel up
    to the rounding of the separate accumulation."""
    case = _case((33, 17, 10))
    case.scheme.reconstruction = rec
    case.scheme.inviscid_scheme = flux
    ref = OracleRun(case)
    ref.initialize()
    scale = ref.flux_scale()
    s, blocks = _gpu(case)
    s.initialize()
    s.compute_rhs()
    fused = blocks[0].download("dq")
    for d in range(3):
        s.set_tile(d + 3, *vtile)
        assert s.get_tile(d + 3) == vtile
    s.compute_rhs()
    split = blocks[0].download("dq")
    assert max(rhs_errors(split, ref.blocks[0].arrays["dq"], scale)) <= RHS_TOL
    assert max(rhs_errors(split, fused, scale)) <= 1e-13
    for d in range(3):
        s.set_tile(d + 3, 0, 0)
        assert s.get_tile(d + 3) == (0, 0)
    s.compute_rhs()
    assert np.array_equal(blocks[0].download("dq"), fused)
    s.close()


def test_flux_halves_add_up():
    """OP_FLUX arg d + 3 (inviscid kernel alone) and d + 6 (viscous kernel
    alone) accumulate to what arg d (the direction's whole flux) adds."""
    import torch

    case = _case((24, 20, 8))
    ref = OracleRun(case)
    ref.initialize()
    scale = ref.flux_scale()
    s, blocks = _gpu(case)
    s.initialize()
    dq = blocks[0].t["dq"]
    for d in range(3):
        dq.zero_()
        s.launch_op(s.OP_FLUX, d)
        torch.cuda.synchronize()
        whole = blocks[0].download("dq")
        dq.zero_()
        s.launch_op(s.OP_FLUX, d + 3)
        s.launch_op(s.OP_FLUX, d + 6)
        torch.cuda.synchronize()
        assert max(rhs_errors(blocks[0].download("dq"), whole, scale)) <= 1e-13, d
    s.close()
