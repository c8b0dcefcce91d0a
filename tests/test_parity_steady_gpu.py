"""GPU parity of the steady path (steady_simulation, src/SteadySim.cuh:
15-137): local time stepping with the explicit update and point-implicit
chemistry (EPI, DA; src/FiniteRateChem.cu:196-432) or DPLUR (src/DPLUR.cuh,
src/DPLUR.cu), against the CPU oracle and against the reference's own CUDA
kernels on the same blocks.

Cases: a stoichiometric H2-air box at 1400 K (chemistry active on the cell
time scale, so EPI / DA / explicit differ), the air vortex with MUSCL + Roe,
and the air box with an isothermal wall (DPLUR zeroes dq on it before every
sweep). Bars: 1e-9 normwise on states and residual histories after the
steps (the RK3 bar)."""
import numpy as np
import pytest

import ostc
import ref_bind
from oracle_bind import OracleRun, normwise

pytestmark = pytest.mark.gpu

VARIANTS = [("premixed", 0, 0), ("premixed", 0, 1), ("premixed", 0, 2), ("premixed", 1, 0), ("premixed", 1, 1),
            ("premixed", 1, 2), ("vortex", 0, None), ("vortex", 1, None), ("wall", 1, None)]


def _case(kind, implicit_method, chem):
    if kind == "premixed":
        base = ostc.case_premixed_box(16, 14, 8)
    elif kind == "vortex":
        base = ostc.case_vortex(20, 16, 6, k_bc="symmetry", reconstruction=2, inviscid_scheme=2)
    else:
        base = ostc.case_bc_box("wall")
    return ostc.make_steady(base, implicit_method=implicit_method, chem_src_method=chem)


def _ids(v):
    return "%s-im%d-chem%s" % v


def _reduction_well_defined(cells):
    nb = (cells + 127) // 128
    v1, v2 = cells - (nb - 1) * 128, nb
    return all(v == 128 or v % 32 for v in (v1, v2))


def _compare(blocks, got_fn, n_spec):
    for b in range(len(blocks)):
        for name in ("bv", "sv") if n_spec else ("bv",):
            err = normwise(blocks[b].download(name), got_fn(name, b))
            assert max(err) <= 1e-9, (b, name, err)


@pytest.mark.parametrize("variant", VARIANTS, ids=_ids)
def test_steady_matches_oracle(variant):
    case = _case(*variant)
    n = 8
    o = OracleRun(case)
    o.initialize()
    res_o = o.steady_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g = s.steady_steps(n, history=True)
    _compare(blocks, lambda name, b: o.blocks[b].arrays[name], case.blocks[0].n_spec)
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9


@pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("variant", VARIANTS, ids=_ids)
def test_steady_matches_reference_build(variant):
    case = _case(*variant)
    assert all(_reduction_well_defined(b.mx * b.my * b.mz) for b in case.blocks)
    n = 8
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    res_r = r.steady_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g = s.steady_steps(n, history=True)
    _compare(blocks, lambda name, b: r.download(name, b), case.blocks[0].n_spec)
    assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9


def test_point_implicit_treatments_differ_on_reacting_box():
    """EPI, DA and the explicit update give different states on the reacting
    box (the case exercises the chemical Jacobians), each matching its oracle."""
    out = {}
    for chem in (0, 1, 2):
        case = _case("premixed", 0, chem)
        s, blocks = case.solver()
        s.initialize()
        s.steady_steps(8)
        out[chem] = blocks[0].download("sv")
    assert np.max(np.abs(out[1] - out[0])) > 1e-8
    assert np.max(np.abs(out[2] - out[0])) > 1e-8
    assert np.max(np.abs(out[1] - out[2])) > 1e-8
