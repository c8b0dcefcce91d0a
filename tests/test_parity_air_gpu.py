"""GPU parity of the single-species air path (AWENO-5 + AUSM+, laminar
viscous, SSPRK3) against the CPU oracle, through the C ABI.

Tolerances: one RHS evaluation must agree with the oracle to 1e-11
normwise per variable, max|d dq_l| / max(max|dq_l|, 1e-2 * F_l), where F_l
is the largest face flux of variable l (tests/oracle_bind.py: rhs_errors).
FP64 on both sides; the difference comes from FMA contraction and libm
last-ulp differences, which scale with the face fluxes that dq is a
difference of.
Multi-step histories drift by rounding amplification and are held to 1e-9.
"""
import numpy as np
import pytest

import ostc
from oracle_bind import OracleRun, normwise, rhs_errors

RHS_TOL = 1e-11
STEP_TOL = 1e-9

pytestmark = pytest.mark.gpu


def _gpu_solver(case):
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    return ostc.Solver(case.scheme, case.mech, blocks, case.faces), blocks


def _rhs_pair(case):
    ref = OracleRun(case)
    ref.initialize()
    ref.scale = ref.flux_scale()
    s, blocks = _gpu_solver(case)
    s.initialize()
    s.compute_rhs()
    import torch

    torch.cuda.synchronize()
    return ref, s, blocks


@pytest.mark.parametrize("k_bc", ["periodic", "symmetry"])
@pytest.mark.parametrize("shape", [(32, 24, 8), (45, 19, 11)])
def test_initialize_matches(shape, k_bc):
    case = ostc.case_vortex(*shape, k_bc=k_bc)
    ref = OracleRun(case)
    ref.initialize()
    s, blocks = _gpu_solver(case)
    s.initialize()
    hb = ref.blocks[0].arrays
    for name in ("bv", "cv", "vel", "acoustic_speed", "mul", "thermal_conductivity", "mach"):
        got = blocks[0].download(name)
        assert np.max(np.abs(got - hb[name])) <= 1e-12 * max(1.0, np.max(np.abs(hb[name]))), name


@pytest.mark.parametrize("k_bc", ["periodic", "symmetry"])
@pytest.mark.parametrize("shape", [(32, 24, 8), (45, 19, 11), (64, 64, 8)])
def test_rhs_matches_oracle(shape, k_bc):
    case = ostc.case_vortex(*shape, k_bc=k_bc)
    ref, s, blocks = _rhs_pair(case)
    err = rhs_errors(blocks[0].download("dq"), ref.blocks[0].arrays["dq"], ref.scale)
    assert max(err) <= RHS_TOL, err


@pytest.mark.parametrize("tiles", [((2, 1), (4, 1), (4, 1)), ((8, 3), (8, 5), (4, 2)), ((4, 2), (2, 3), (8, 1))])
def test_rhs_independent_of_tile_shape(tiles):
    case = ostc.case_vortex(40, 30, 9)
    ref, s, blocks = _rhs_pair(case)
    base = blocks[0].download("dq")
    for d, (r, c) in enumerate(tiles):
        s.set_tile(d, r, c)
    s.compute_rhs()
    assert np.array_equal(blocks[0].download("dq"), base)


def test_dt_matches_oracle():
    case = ostc.case_vortex(32, 24, 8)
    ref, s, blocks = _rhs_pair(case)
    assert abs(s.global_time_step() - ref.global_time_step()) <= 1e-14 * ref.global_time_step()


@pytest.mark.parametrize("k_bc", ["periodic", "symmetry"])
def test_rk3_history_matches_oracle(k_bc):
    case = ostc.case_vortex(32, 24, 8, k_bc=k_bc)
    n = 10
    ref = OracleRun(case)
    ref.initialize()
    res_o, dt_o = ref.rk3_steps(n)
    s, blocks = _gpu_solver(case)
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= STEP_TOL
    assert np.max(np.abs(res_g - res_o) / res_o) <= STEP_TOL
    err = normwise(blocks[0].download("bv"), ref.blocks[0].arrays["bv"])
    assert max(err) <= STEP_TOL, err


def test_stage_by_stage_equals_graph():
    case = ostc.case_vortex(24, 20, 8)
    s1, b1 = _gpu_solver(case)
    s1.initialize()
    s1.rk3_steps(2)
    s2, b2 = _gpu_solver(case)
    s2.initialize()
    import torch

    for _ in range(2):
        b2[0].t["qn"].copy_(b2[0].t["cv"])
        for rk in range(3):
            s2.rk3_stage(rk)
    torch.cuda.synchronize()
    assert np.array_equal(b1[0].download("bv"), b2[0].download("bv"))


def test_deterministic_rerun():
    case = ostc.case_vortex(32, 24, 8)
    outs = []
    for _ in range(2):
        s, blocks = _gpu_solver(case)
        s.initialize()
        s.rk3_steps(3)
        outs.append(blocks[0].download("cv"))
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("rec,flux", [(2, 2), (3, 2), (1, 2), (2, 1), (3, 1), (2, 3), (2, 4)])
def test_rhs_other_air_schemes(rec, flux):
    # Roe flux-difference splitting (inviscid_type 2), Lax-Friedrichs, AUSM+ and HLLC on
    # primitive-variable reconstructions
    case = ostc.case_vortex(36, 28, 9, reconstruction=rec, inviscid_scheme=flux)
    ref, s, blocks = _rhs_pair(case)
    err = rhs_errors(blocks[0].download("dq"), ref.blocks[0].arrays["dq"], ref.scale)
    assert max(err) <= RHS_TOL, err


def test_rk3_history_roe():
    case = ostc.case_vortex(32, 24, 8, reconstruction=2, inviscid_scheme=2)
    ref = OracleRun(case)
    ref.initialize()
    res_o, dt_o = ref.rk3_steps(8)
    s, blocks = _gpu_solver(case)
    s.initialize()
    res_g, dt_g = s.rk3_steps(8, history=True)
    assert np.max(np.abs(res_g - res_o) / res_o) <= STEP_TOL
    assert max(normwise(blocks[0].download("bv"), ref.blocks[0].arrays["bv"])) <= STEP_TOL
