"""Wall, far-field, back-pressure and subsonic-inflow boundary conditions:
GPU vs the CPU oracle and vs the reference build (BoundCond.cuh:212-671),
air and 9-species mixture. Tolerances as in the other parity tests."""
import numpy as np
import pytest

import ostc
import ref_bind
from oracle_bind import OracleRun, normwise, rhs_errors

pytestmark = pytest.mark.gpu


def _mixture_wall_farfield(shape=(30, 26, 10)):
    c = ostc.case_mixing_layer(*shape, full_host=True)
    ng = c.blocks[0].ngg
    ext = shape
    m = c.mech
    Y = np.zeros(m.n_spec)
    Y[m.names.index("O2")], Y[m.names.index("N2")] = 0.233, 0.767
    ff = ostc.farfield_state(2.0, 1500.0, 101325.0, mech=m, Y=Y)
    c.faces = [ostc.bc_face(0, ostc.BC_OUTFLOW, 0, -1, ext, ng), ostc.bc_face(0, ostc.BC_OUTFLOW, 0, 1, ext, ng),
               ostc.bc_face(0, ostc.BC_WALL, 1, -1, ext, ng, dict(wall_isothermal=1, wall_temperature=300.0)),
               ostc.bc_face(0, ostc.BC_FARFIELD, 1, 1, ext, ng, ff),
               ostc.bc_face(0, ostc.BC_OUTFLOW, 2, -1, ext, ng), ostc.bc_face(0, ostc.BC_OUTFLOW, 2, 1, ext, ng)]
    return c


CASES = {"air_wall_farfield": lambda: ostc.case_bc_box("wall_farfield"),
         "air_subsonic": lambda: ostc.case_bc_box("subsonic"),
         "mixture_wall_farfield": _mixture_wall_farfield}


@pytest.mark.parametrize("name", list(CASES))
def test_rhs_and_history_vs_oracle(name):
    case = CASES[name]()
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale()
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    s.compute_rhs()
    assert max(rhs_errors(blocks[0].download("dq"), o.blocks[0].arrays["dq"], scale)) <= 1e-11
    res_o, dt_o = o.rk3_steps(8)
    res_g, dt_g = s.rk3_steps(8, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert max(normwise(blocks[0].download("bv"), o.blocks[0].arrays["bv"])) <= 1e-9


@pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", list(CASES))
def test_rhs_and_history_vs_reference_build(name):
    case = CASES[name]()
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    r.compute_rhs()
    dq_ref = r.download("dq")
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale()
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    s.compute_rhs()
    assert max(rhs_errors(blocks[0].download("dq"), dq_ref, scale)) <= 1e-11
    _, dt_r = r.rk3_steps(8)
    _, dt_g = s.rk3_steps(8, history=True)
    assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
    assert max(normwise(blocks[0].download("bv"), r.download("bv"))) <= 1e-9
