"""Known-answer and invariant tests of the CPU oracle (no GPU)."""
import ctypes as C

import numpy as np
import pytest

import chemdata
import ostc
from oracle_bind import OracleRun, oracle


@pytest.fixture(scope="module")
def mech():
    return chemdata.h2_air_9sp()


def _param(mech):
    s = ostc.Scheme(mix_model=ostc.MIX_FR)
    return ostc.make_param(s, mech)


def test_species_mass_conservation(mech):
    p, keep = _param(mech)
    rng = np.random.default_rng(1)
    for _ in range(20):
        Y = rng.uniform(0, 1, mech.n_spec)
        Y /= Y.sum()
        T = rng.uniform(800, 2500)
        om = (C.c_double * mech.n_spec)()
        y = (C.c_double * mech.n_spec)(*Y)
        assert oracle().oracle_chemical_source(C.byref(p), 0.3, T, y, om) == 0
        om = np.array(om)
        assert abs(om.sum()) <= 1e-10 * np.abs(om).max()


def test_element_conservation(mech):
    # H, O, N atoms in each species of the 9-species set
    comp = {"H2": (2, 0, 0), "H": (1, 0, 0), "O2": (0, 2, 0), "O": (0, 1, 0), "OH": (1, 1, 0), "HO2": (1, 2, 0),
            "H2O2": (2, 2, 0), "H2O": (2, 1, 0), "N2": (0, 0, 2)}
    A = np.array([comp[n] for n in mech.names], dtype=float)
    p, keep = _param(mech)
    Y = np.full(mech.n_spec, 1.0 / mech.n_spec)
    om = (C.c_double * mech.n_spec)()
    oracle().oracle_chemical_source(C.byref(p), 0.5, 1800.0, (C.c_double * mech.n_spec)(*Y), om)
    rates = np.array(om) / mech.tables["mw"]
    for e in range(3):
        tot = np.abs(A[:, e] * rates).sum()
        assert abs((A[:, e] * rates).sum()) <= 1e-10 * max(tot, 1e-300)


def test_enthalpy_continuous_at_tmid(mech):
    p, keep = _param(mech)
    ns = mech.n_spec
    h0, c0 = (C.c_double * ns)(), (C.c_double * ns)()
    h1, c1 = (C.c_double * ns)(), (C.c_double * ns)()
    oracle().oracle_enthalpy_cp(C.byref(p), 1000.0 - 1e-9, h0, c0)
    oracle().oracle_enthalpy_cp(C.byref(p), 1000.0 + 1e-9, h1, c1)
    h0, h1 = np.array(h0), np.array(h1)
    assert np.all(np.abs(h1 - h0) <= 2e-3 * np.maximum(np.abs(h0), 1e5))


def test_enthalpy_linear_below_tlow(mech):
    # below T_low, h continues linearly with the slope cp(T_low) (Thermo.cu:8-15)
    p, keep = _param(mech)
    ns = mech.n_spec
    hs = []
    for T in (100.0, 150.0):
        h, c = (C.c_double * ns)(), (C.c_double * ns)()
        oracle().oracle_enthalpy_cp(C.byref(p), T, h, c)
        hs.append((np.array(h), np.array(c)))
    (h1, c1), (h2, c2) = hs
    assert np.allclose(h2 - h1, c1 * 50.0, rtol=1e-12, atol=1e-6)


def test_transport_positive(mech):
    p, keep = _param(mech)
    ns = mech.n_spec
    Y = np.full(ns, 1.0 / ns)
    mu, k = C.c_double(), C.c_double()
    rd = (C.c_double * ns)()
    oracle().oracle_transport(C.byref(p), 0.4, 101325.0, 900.0, (C.c_double * ns)(*Y), C.byref(mu), C.byref(k), rd)
    assert 1e-6 < mu.value < 1e-3 and 1e-3 < k.value < 1.0 and np.all(np.array(rd) > 0)


@pytest.mark.parametrize("rec", [1, 2, 3])
def test_freestream_preserved_cartesian(rec):
    # uniform flow on an unwarped grid: every face flux is the same, dq = 0
    case = ostc.case_vortex(16, 12, 8)
    case.scheme.reconstruction = rec
    case.scheme.inviscid_scheme = 3
    b = case.blocks[0]
    x, y, z = ostc.grid_coordinates(16, 12, 8, b.ngg + 1, 1e-3, warp=0.0)
    ostc.fill_metric(b, x, y, z)
    inf = ostc.air_state(2.0, 300.0, 101325.0)
    bv = b.arrays["bv"]
    bv[0], bv[1], bv[2], bv[3], bv[4], bv[5] = inf["density"], inf["u"], 0, 0, inf["pressure"], 300.0
    case.faces = [f for f in case.faces if f.type_label == ostc.BC_PERIODIC]
    r = OracleRun(case)
    r.initialize()
    r.compute_rhs()
    dq = r.blocks[0].arrays["dq"]
    assert np.abs(dq[:, :, :, 2:-2]).max() <= 1e-9 * inf["density"] * inf["u"] ** 2


def test_oracle_thread_count_invariant():
    case = ostc.case_vortex(20, 16, 8)
    outs = []
    for t in (1, 4):
        oracle().oracle_set_threads(t)
        r = OracleRun(case)
        r.initialize()
        r.rk3_steps(2)
        outs.append(r.blocks[0].arrays["bv"].copy())
    assert np.array_equal(outs[0], outs[1])


def test_ssprk3_is_third_order_on_linear_ode():
    # cv_t = dq/J with dq = -lam*cv*J reduces to the SSPRK3 update of y' = -lam y
    lam, T = 3.0, 1.0
    errs = []
    for n in (20, 40, 80):
        dt = T / n
        y = 1.0
        for _ in range(n):
            y1 = y + dt * (-lam * y)
            y2 = 0.75 * y + 0.25 * y1 + 0.25 * dt * (-lam * y1)
            y = y / 3.0 + 2.0 / 3.0 * y2 + 2.0 / 3.0 * dt * (-lam * y2)
        errs.append(abs(y - np.exp(-lam * T)))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 2.8)
