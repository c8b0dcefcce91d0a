"""Known-answer properties of the FP64 point-implicit chemistry integrator
(the oracle's restatement; CPU only): one linearised backward-Euler step of
d(rho Y)/dt = omega at constant density and internal energy.

* mass: every reaction conserves mass, so the columns of J sum to zero and
  sum_k dY_k = 0 to round-off;
* elements: sum_k a_ek dY_k / W_k = 0 for H, O, N;
* energy: e(T + dT, Y + dY) = e(T, Y) with e = sum Y h(T) - R_u T sum(Y/W);
* consistency: dY / dt -> omega / rho as dt -> 0.
"""
import numpy as np
import pytest

import chemdata
import ostc
from oracle_bind import chem_point_implicit, oracle
import ctypes as C


@pytest.fixture(scope="module")
def mech():
    return chemdata.h2_air_9sp()


@pytest.fixture(scope="module")
def states(mech):
    return ostc.sample_chem_states(mech, 400, seed=5)


def _energy(mech, T, Y):
    prm, keep = ostc.make_param(ostc.Scheme(mix_model=ostc.MIX_FR), mech)
    ns = mech.n_spec
    W = mech.tables["mw"]
    out = np.empty(T.size)
    h = np.zeros(ns)
    cp = np.zeros(ns)
    for q in range(T.size):
        oracle().oracle_enthalpy_cp(C.byref(prm), float(T[q]), h.ctypes.data_as(C.POINTER(C.c_double)),
                                    cp.ctypes.data_as(C.POINTER(C.c_double)))
        out[q] = np.dot(Y[:, q], h) - ostc.R_U * T[q] * np.sum(Y[:, q] / W)
    return out


def test_mass_conserved(mech, states):
    T, p, Y, dt = states
    dY, dT = chem_point_implicit(mech, T, p, Y, dt)
    assert np.all(np.isfinite(dT))
    assert np.max(np.abs(dY.sum(axis=0))) <= 1e-13


def test_elements_conserved(mech, states):
    T, p, Y, dt = states
    dY, _ = chem_point_implicit(mech, T, p, Y, dt)
    W = mech.tables["mw"]
    for el, a in ostc.species_elements(mech.names).items():
        moles = (a[:, None] * dY / W[:, None]).sum(axis=0)
        scale = (a[:, None] * np.abs(dY) / W[:, None]).sum(axis=0) + 1e-300
        assert np.max(np.abs(moles) / scale) <= 1e-10, el


def test_internal_energy_conserved(mech, states):
    T, p, Y, dt = states
    dY, dT = chem_point_implicit(mech, T, p, Y, dt)
    e0 = _energy(mech, T, Y)
    e1 = _energy(mech, T + dT, Y + dY)
    # the Newton solve stops at |1 - T1/T| <= 1e-13: e agrees to cp * T * 1e-13
    assert np.max(np.abs(e1 - e0) / (np.abs(e0) + 1e6)) <= 1e-10


def test_small_step_limit_is_the_source(mech, states):
    T, p, Y, dt = states
    dt_small = np.full_like(T, 1e-14)
    dY, _ = chem_point_implicit(mech, T, p, Y, dt_small)
    prm, keep = ostc.make_param(ostc.Scheme(mix_model=ostc.MIX_FR), mech)
    W = mech.tables["mw"]
    om = np.zeros(mech.n_spec)
    worst = 0.0
    for q in range(0, T.size, 20):
        rho = p[q] / (ostc.R_U * T[q] * np.sum(Y[:, q] / W))
        y = np.ascontiguousarray(Y[:, q])
        oracle().oracle_chemical_source(C.byref(prm), rho, float(T[q]), y.ctypes.data_as(C.POINTER(C.c_double)),
                                        om.ctypes.data_as(C.POINTER(C.c_double)))
        rate = dY[:, q] / 1e-14
        worst = max(worst, np.max(np.abs(rate - om / rho)) / (np.max(np.abs(om / rho)) + 1e-300))
    assert worst <= 1e-6


def test_stiff_step_damps_the_explicit_overshoot(mech):
    """At dt = 1e-5 s in hot mixtures the explicit update dY = dt omega / rho
    drives mass fractions far out of [0, 1]; the point-implicit step (one
    linearised backward-Euler step, not positivity-preserving) stays within
    a small fraction of that excursion."""
    T, p, Y, dt = ostc.sample_chem_states(mech, 200, seed=9, T_range=(1500, 2500), dt_range=(1e-5, 1e-5))
    dY, dT = chem_point_implicit(mech, T, p, Y, dt)
    assert np.all(np.isfinite(dT))
    prm, keep = ostc.make_param(ostc.Scheme(mix_model=ostc.MIX_FR), mech)
    W = mech.tables["mw"]
    om = np.zeros(mech.n_spec)
    dY_exp = np.zeros_like(dY)
    for q in range(T.size):
        rho = p[q] / (ostc.R_U * T[q] * np.sum(Y[:, q] / W))
        y = np.ascontiguousarray(Y[:, q])
        oracle().oracle_chemical_source(C.byref(prm), rho, float(T[q]), y.ctypes.data_as(C.POINTER(C.c_double)),
                                        om.ctypes.data_as(C.POINTER(C.c_double)))
        dY_exp[:, q] = dt[q] * om / rho
    under_imp = max(0.0, -(Y + dY).min())
    under_exp = max(0.0, -(Y + dY_exp).min())
    assert under_exp > 1.0
    assert under_imp < 0.05 * under_exp
