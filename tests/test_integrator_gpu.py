"""GPU parity of the FP64 point-implicit chemistry integrator
(ostc_chem_point_implicit) against the oracle's restatement, on seeded
states spanning the surrogate's training envelope (T 300-3000 K, p 0.5-3
atm, dt 1e-9-1e-7 s) and on stiff steps (dt 1e-5 s). Bar: 1e-9 per species
relative to the largest |dY| of that species, 1e-9 relative on dT, and the
same states flagged (NaN dT) where the energy solve has no root."""
import numpy as np
import pytest

import ostc
from oracle_bind import chem_point_implicit, normwise

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    case = ostc.case_premixed_box(8, 8, 4)
    s, blocks = case.solver()
    yield s, case.mech
    s.close()


@pytest.mark.parametrize("dt_range", [(1e-9, 1e-7), (1e-5, 1e-5)], ids=["envelope", "stiff"])
def test_integrator_matches_oracle(solver, dt_range):
    import torch

    s, mech = solver
    T, p, Y, dt = ostc.sample_chem_states(mech, 20000, seed=3, dt_range=dt_range)
    dY_o, dT_o = chem_point_implicit(mech, T, p, Y, dt)
    dev = [torch.from_numpy(a).cuda() for a in (T, p, Y, dt)]
    dY, dT = s.chem_point_implicit(*dev)
    torch.cuda.synchronize()
    dY, dT = dY.cpu().numpy(), dT.cpu().numpy()
    # a stiff step can overshoot to negative mass fractions where the energy
    # Newton solve has no root; both sides flag the same states with NaN
    ok = np.isfinite(dT_o)
    assert np.array_equal(np.isfinite(dT), ok)
    assert ok.mean() > 0.99
    assert max(normwise(dY[:, ok], dY_o[:, ok])) <= 1e-9
    assert normwise(dT[ok], dT_o[ok], axis_vars=False) <= 1e-9
