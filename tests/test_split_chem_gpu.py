"""Operator-split chemistry in the RK3 step (config chem_mode): the three
flow stages without the chemistry source, then the chemistry of each cell
over the step's dt at constant density and internal energy.

* chem_mode 1 (FP64 point-implicit integrator) against the oracle's
  restatement of the same split step: states, dt and residual histories to
  1e-9 on a reacting premixed box and on the mixing layer;
* chem_mode 2 (learned surrogate + FP64 fallback) with acceptance tests
  that reject every state equals chem_mode 1 to round-off: the fallback
  path is the integrator itself;
* chem_mode 2 with a trained surrogate stays close to chem_mode 1 and
  reports how many states fell back."""
import numpy as np
import pytest

import ostc
import surrogate as S
from oracle_bind import OracleRun, normwise

pytestmark = pytest.mark.gpu


def _premixed(mode):
    c = ostc.case_premixed_box(16, 14, 8, dx=1e-3, T0=1500.0)
    c.scheme.chem_mode = mode
    return c


def _mixing(mode):
    c = ostc.case_mixing_layer(24, 20, 8, dx=1e-3, full_host=True)
    c.scheme.chem_mode = mode
    return c


@pytest.mark.parametrize("build", [_premixed, _mixing], ids=["premixed", "mixing"])
def test_split_fp64_matches_oracle(build):
    case = build(1)
    n = 5
    o = OracleRun(case)
    o.initialize()
    res_o, dt_o = o.rk3_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for name in ("bv", "sv"):
        assert max(normwise(blocks[0].download(name), o.blocks[0].arrays[name])) <= 1e-9, name
    states, fb = s.chem_stats()
    assert states == n * case.cells and fb == 0


@pytest.fixture(scope="module")
def trained():
    case = _premixed(1)
    solver, _ = case.solver()
    sur, sc, log = S.build(solver, case.mech, n_train=600_000, epochs=6, seed=3)
    yield sur, case.mech
    sur.close()


def test_surrogate_rejecting_everything_is_the_fp64_split(trained):
    sur, mech = trained
    S.set_checks(sur, mech, tol_elem=0.0, tol_T=0.0)
    a = _premixed(1)
    b = _premixed(2)
    sa, ba = a.solver()
    sb, bb = b.solver()
    sb.set_chem_surrogate(sur)
    sa.initialize()
    sb.initialize()
    sa.rk3_steps(4)
    sb.rk3_steps(4)
    for name in ("bv", "sv"):
        assert max(normwise(bb[0].download(name), ba[0].download(name))) <= 1e-12, name
    states, fb = sb.chem_stats()
    assert states == 4 * b.cells and fb == states
    S.set_checks(sur, mech)


def test_trained_surrogate_tracks_the_fp64_split(trained):
    sur, mech = trained
    a = _premixed(1)
    b = _premixed(2)
    sa, ba = a.solver()
    sb, bb = b.solver()
    sb.set_chem_surrogate(sur)
    sa.initialize()
    sb.initialize()
    sa.rk3_steps(4)
    sb.rk3_steps(4)
    dT = np.abs(bb[0].download("bv")[5] - ba[0].download("bv")[5]).max()
    dY = np.abs(bb[0].download("sv") - ba[0].download("sv")).max()
    states, fb = sb.chem_stats()
    assert states == 4 * b.cells
    assert dT < 5.0 and dY < 5e-3, (dT, dY, fb / states)
