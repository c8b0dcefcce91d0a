"""GPU parity of k-omega SST with the 9-species H2-air mixture (the
reference's Driver<FR, SST>): the SST source with the mixture's gamma and
cp, the turbulent species diffusivity mut / Sct, k and omega after the
species (i_turb_cv = 5 + n_spec), the wall's mixture viscosity, and the
chemistry and turbulence rows of the steady path. Against the oracle (RHS
1e-11 of the flux scale, histories and states 1e-9) and the reference's own
kernels, on the reacting mixing layer with SST (ostc.case_mixing_layer with
rans_model=2; wall=True puts an isothermal wall at j = 0)."""
import numpy as np
import pytest

import ostc
from oracle_bind import OracleRun, rhs_errors

pytestmark = pytest.mark.gpu


def _case(wall=False, corr=0, periodic=True):
    c = ostc.case_mixing_layer(20, 18, 6, full_host=True, rans_model=2, wall=wall, compressibility_correction=corr)
    if not periodic:  # the reference has no periodic faces (quirk A13)
        for f in c.faces:
            if f.type_label == ostc.BC_PERIODIC:
                f.type_label = ostc.BC_OUTFLOW
    return c


def _errors(got, ref):
    """normwise per plane, velocity components sharing the largest one's scale"""
    den = [float(np.max(np.abs(ref[l]))) for l in range(ref.shape[0])]
    vel = max(den[1:4]) if ref.shape[0] == 6 else None
    return [float(np.max(np.abs(got[l] - ref[l]))) / ((vel if vel and 1 <= l <= 3 else den[l]) or 1.0)
            for l in range(ref.shape[0])]


@pytest.mark.parametrize("wall,corr", [(False, 0), (True, 0), (True, 1), (True, 3)])
def test_mixture_sst_rhs_matches_oracle(wall, corr):
    case = _case(wall, corr)
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale(0)
    o.compute_rhs()
    s, blocks = case.solver()
    s.initialize()
    mo = o.blocks[0].arrays["mut"]
    assert np.max(np.abs(blocks[0].download("mut") - mo)) <= 1e-12 * np.max(np.abs(mo))
    s.compute_rhs()
    err = rhs_errors(blocks[0].download("dq"), o.blocks[0].arrays["dq"], scale)
    assert max(err) <= 1e-11, err
    for arr in ("mut", "turb_therm_cond"):
        ref = o.blocks[0].arrays[arr]
        assert np.max(np.abs(blocks[0].download(arr) - ref)) <= 1e-12 * np.max(np.abs(ref)), arr
    s.close()


@pytest.mark.parametrize("wall", [False, True])
def test_mixture_sst_history_matches_oracle(wall):
    case = _case(wall)
    n = 5
    o = OracleRun(case)
    o.initialize()
    res_o, dt_o = o.rk3_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    assert max(_errors(blocks[0].download("bv"), o.blocks[0].arrays["bv"])) <= 1e-9
    assert max(_errors(blocks[0].download("sv"), o.blocks[0].arrays["sv"])) <= 1e-9
    ref = o.blocks[0].arrays["mut"]
    assert np.max(np.abs(blocks[0].download("mut") - ref)) <= 1e-9 * np.max(np.abs(ref))
    s.close()


@pytest.mark.skipif(not __import__("ref_bind").available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("wall", [False, True])
def test_mixture_sst_matches_reference_build(wall):
    """Driver<FR, SST>'s own kernels: initial mut, one RHS (1e-11) and 5 RK3
    steps at the CFL dt (dt, residuals, states to 1e-9)"""
    import ref_bind

    case = _case(wall, periodic=False)
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale(0)
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    s, blocks = case.solver()
    s.initialize()
    mr = r.download("mut")
    assert np.max(np.abs(blocks[0].download("mut") - mr)) <= 1e-12 * np.max(np.abs(mr))
    r.compute_rhs()
    s.compute_rhs()
    assert max(rhs_errors(blocks[0].download("dq"), r.download("dq"), scale)) <= 1e-11
    s.close()
    n = 5
    r2 = ref_bind.RefCudaRun(case)
    r2.initialize()
    res_r, dt_r = r2.rk3_steps(n)
    s2, blocks2 = case.solver()
    s2.initialize()
    res_g, dt_g = s2.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
    assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    assert max(_errors(blocks2[0].download("bv"), r2.download("bv"))) <= 1e-9
    assert max(_errors(blocks2[0].download("sv"), r2.download("sv"))) <= 1e-9
    s2.close()


@pytest.mark.parametrize("implicit_method,turb_implicit,chem", [(0, 1, 1), (0, 0, 2), (1, 1, 1), (1, 0, 2),
                                                                (1, 1, 0)])
def test_mixture_sst_steady(implicit_method, turb_implicit, chem):
    """the steady path of Driver<FR, SST>: explicit (EPI / DA chemistry, then
    the SST point-implicit sources) or DPLUR with both in its diagonal; 4
    iterations against the oracle and the reference's kernels"""
    import ref_bind

    base = _case(True, periodic=False)
    base.scheme.turb_implicit = turb_implicit
    case = ostc.make_steady(base, implicit_method=implicit_method, chem_src_method=chem, dplur_inner_step=2)
    n = 4
    o = OracleRun(case)
    o.initialize()
    res_o = o.steady_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g = s.steady_steps(n, history=True)
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    assert max(_errors(blocks[0].download("bv"), o.blocks[0].arrays["bv"])) <= 1e-9
    assert max(_errors(blocks[0].download("sv"), o.blocks[0].arrays["sv"])) <= 1e-9
    s.close()
    if not ref_bind.available():
        return
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    res_r = r.steady_steps(n)
    assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    s2, blocks2 = case.solver()
    s2.initialize()
    s2.steady_steps(n)
    assert max(_errors(blocks2[0].download("bv"), r.download("bv"))) <= 1e-9
    assert max(_errors(blocks2[0].download("sv"), r.download("sv"))) <= 1e-9
    s2.close()
