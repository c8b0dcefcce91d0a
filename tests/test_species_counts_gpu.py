"""Mechanisms of every species count up to MAX_SPEC_NUMBER (20, the
reference build's CMakeLists.txt:13-19), each on its own compile-time build
(kernels_ns_*.cu, flux_ns_*.cu):

* the reference's own non-reacting set of input_files/chemistry/
  H2_mech_mixing.inp (H2, H2O, O2, N2; MixtureModel::Mixture);
* a 7-species reacting subset of the H2-air mechanism (the 8 reactions
  among H2, H, O2, O, OH, H2O, N2);
* 3 species, and 12 and 20 species made of the H2-air mechanism plus inert
  copies of N2 that carry part of its mass fraction.

RHS and short histories against the CPU oracle and, where the reference
build can run the set, against the reference's own kernels.
"""
import numpy as np
import pytest

import chemdata
import ostc
import ref_bind
from oracle_bind import OracleRun, normwise, rhs_errors

pytestmark = pytest.mark.gpu


def _mech(name):
    m9 = chemdata.h2_air_9sp()
    if name == "mixing4":
        return chemdata.h2_mixing_4sp()
    if name == "sub3":
        return chemdata.subset(m9, ["H2", "O2", "N2"])
    if name == "sub7":
        return chemdata.subset(m9, ["H2", "H", "O2", "O", "OH", "H2O", "N2"])
    if name == "inert12":
        return chemdata.with_inert_copies(m9, "N2", 3)
    return chemdata.with_inert_copies(m9, "N2", 11)  # 20 species


def _case(name, shape=(24, 20, 8), mix_model=None, outflow=False):
    mech = _mech(name)
    c = ostc.case_mixing_layer(*shape, dx=1e-3, full_host=True, mech=mech, mix_model=mix_model)
    names = mech.names
    copies = [i for i, n in enumerate(names) if n.startswith("N2_")]
    if copies:  # the copies carry equal shares of the nitrogen
        sv = c.blocks[0].arrays["sv"]
        n2 = names.index("N2")
        share = sv[n2] / (len(copies) + 1)
        sv[n2] = share
        for i in copies:
            sv[i] = share
    if outflow:  # the reference has no periodic boundary
        for f in c.faces:
            if f.type_label == ostc.BC_PERIODIC:
                f.type_label = ostc.BC_OUTFLOW
    return c


NAMES = ["mixing4", "sub3", "sub7", "inert12", "inert20"]


@pytest.mark.parametrize("name", NAMES)
def test_rhs_and_history_match_oracle(name):
    case = _case(name)
    assert case.mech.n_spec == {"mixing4": 4, "sub3": 3, "sub7": 7, "inert12": 12, "inert20": 20}[name]
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale()
    o2 = OracleRun(case)
    o2.initialize()
    o2.compute_rhs()
    blocks = [ostc.DeviceBlock(b) for b in case.blocks]
    s = ostc.Solver(case.scheme, case.mech, blocks, case.faces)
    s.initialize()
    s.compute_rhs()
    err = rhs_errors(blocks[0].download("dq"), o2.blocks[0].arrays["dq"], scale)
    assert max(err) <= 1e-11, err
    res_o, dt_o = o2.rk3_steps(5)
    s.initialize()
    res_g, dt_g = s.rk3_steps(5, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for nm in ("bv", "sv"):
        assert max(normwise(blocks[0].download(nm), o2.blocks[0].arrays[nm])) <= 1e-9, nm
    s.close()


@pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", ["mixing4", "sub7", "inert20"])
def test_history_matches_reference_build(name):
    # the reference build runs finite-rate chemistry for every mixture here: the
    # non-reacting set as finite rate with no reactions (its source is zero)
    case = _case(name, shape=(30, 26, 10), mix_model=ostc.MIX_FR, outflow=True)
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
    r2 = ref_bind.RefCudaRun(case)
    r2.initialize()
    res_r, dt_r = r2.rk3_steps(10)
    s.initialize()
    res_g, dt_g = s.rk3_steps(10, history=True)
    assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
    assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    for nm in ("bv", "sv"):
        assert max(normwise(blocks[0].download(nm), r2.download(nm))) <= 1e-9, nm
    s.close()


def test_mixture_and_reaction_free_finite_rate_agree():
    """The non-reacting set as MixtureModel::Mixture and as finite-rate
    chemistry without reactions: the same right-hand side"""
    a = _case("mixing4", mix_model=ostc.MIX_MIXTURE)
    b = _case("mixing4", mix_model=ostc.MIX_FR)
    out = []
    for c in (a, b):
        blocks = [ostc.DeviceBlock(x) for x in c.blocks]
        s = ostc.Solver(c.scheme, c.mech, blocks, c.faces)
        s.initialize()
        s.compute_rhs()
        out.append(blocks[0].download("dq"))
        s.close()
    assert np.array_equal(out[0], out[1])
