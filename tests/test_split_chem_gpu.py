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


# ---------------------------------------------------------------------------
# the surrogate trained on runs of the layer, judged on a layer it never saw
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def trained_on_runs():
    lab = ostc.case_premixed_box(8, 8, 4)
    solver, _ = lab.solver()
    traj = S.trajectory_states(600_000, size=(48, 48, 48), seeds=(5, 6), steps=20, every=5, seed=3)
    sur, sc, log = S.build(solver, lab.mech, n_train=600_000, epochs=12, seed=3, extra_states=traj)
    yield solver, sur, lab.mech
    sur.close()
    solver.close()


def _held_out(mode):
    c = ostc.case_mixing_layer(64, 64, 64, seed=99)  # another noise seed and size than the training runs
    c.scheme.chem_mode = mode
    return c


def test_surrogate_on_held_out_trajectory(trained_on_runs):
    """10 RK3 steps of the learned split against the FP64 split from the same
    state on the held-out layer: the final fields agree to the bar set for the
    learned chemistry (max |dT| < 1 K, max |dY_k| < 1e-4) with at most 5 % of
    the states falling back to the integrator."""
    solver, sur, mech = trained_on_runs
    a, b = _held_out(1), _held_out(2)
    sa, ba = a.solver()
    sb, bb = b.solver()
    sb.set_chem_surrogate(sur)
    sa.initialize()
    sb.initialize()
    sa.rk3_steps(10)
    sb.rk3_steps(10)
    dT = np.abs(bb[0].download("bv")[5] - ba[0].download("bv")[5]).max()
    dY = np.abs(bb[0].download("sv") - ba[0].download("sv")).max()
    states, fb = sb.chem_stats()
    print("held-out trajectory: max |dT| %.3g K, max |dY| %.3g, fallback %.4f" % (dT, dY, fb / states))
    assert states == 10 * b.cells
    assert dT < 1.0 and dY < 1e-4, (dT, dY, fb / states)
    assert fb <= 0.05 * states, fb / states
    sa.close()
    sb.close()


def test_surrogate_gain_over_the_integrator(trained_on_runs):
    """What the trained network gains over the method without it: the learned
    chemistry step (network, checks and FP64 fallback) against the FP64
    point-implicit integrator on the same held-out states (the cells of the
    held-out layer at its time step): less device time per state, and every
    state within 1 K and 1e-4 of the integrator's increment."""
    import torch

    solver, sur, mech = trained_on_runs
    c = _held_out(1)
    s, blocks = c.solver()
    s.initialize()
    _, dts = s.rk3_steps(3, history=True)
    g = c.blocks[0].ngg
    bv, sv = blocks[0].t["bv"], blocks[0].t["sv"]
    T = bv[5, g:-g, g:-g, g:-g].reshape(-1).contiguous()
    p = bv[4, g:-g, g:-g, g:-g].reshape(-1).contiguous()
    Y = sv[:, g:-g, g:-g, g:-g].reshape(sv.shape[0], -1).contiguous()
    dt = torch.full_like(T, float(dts[-1]))
    eT, eY, nfb = S.errors(solver, sur, T, p, Y, dt)
    ms = {}
    for name, fn in (("surrogate", lambda: solver.chem_surrogate(sur, T, p, Y, dt)),
                     ("integrator", lambda: solver.chem_point_implicit(T, p, Y, dt))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms[name] = e0.elapsed_time(e1) / 5
    print("chemistry step of %d states: surrogate %.3f ms, FP64 integrator %.3f ms (%.2fx), fallback %d, "
          "max |dT| %.3g K, max |dY| %.3g" % (T.numel(), ms["surrogate"], ms["integrator"],
                                             ms["integrator"] / ms["surrogate"], nfb, float(eT.max()), float(eY.max())))
    assert float(eT.max()) < 1.0 and float(eY.max()) < 1e-4
    assert ms["surrogate"] < ms["integrator"], ms
    s.close()
