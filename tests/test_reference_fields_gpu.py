"""The drop-in at work: this library run on the reference's own device
arrays. The reference build (oracle/_ref, the reference's sources compiled
for sm_100a) allocates and initialises its DZone; the maintainer's shim
(include/ostc_reference_shim.h, compiled against the reference's Field.h
inside that build) turns the DZone into ostc_zone records; a context
created on them computes the right-hand side and RK3 steps in the
reference's arrays, which then match the reference's own kernels on a copy
of the same fields (RHS 1e-11 of the flux scale, states and histories
1e-9)."""
import numpy as np
import pytest

import ostc
import ref_bind
from oracle_bind import OracleRun, normwise, rhs_errors
from test_parity_refcuda_gpu import _reduction_well_defined

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")]


class _ViewBlock:
    """a block of the reference build seen through the shim"""

    def __init__(self, run, b):
        self.run, self.b = run, b
        hb = run.blocks[b]
        self.mx, self.my, self.mz, self.ngg = hb.mx, hb.my, hb.mz, hb.ngg

    def zone(self):
        return self.run.zone_view(self.b)


def _outflow(case):
    for f in case.faces:  # the reference has no periodic boundary
        if f.type_label == ostc.BC_PERIODIC:
            f.type_label = ostc.BC_OUTFLOW
    return case


CASES = {
    "mixing": lambda: _outflow(ostc.case_mixing_layer(30, 26, 10, dx=1e-3, full_host=True)),
    "vortex_aweno": lambda: _outflow(ostc.case_vortex(40, 32, 10, k_bc="symmetry")),
}


@pytest.mark.parametrize("name", list(CASES))
def test_library_on_the_reference_fields(name):
    case = CASES[name]()
    host = ref_bind.RefCudaRun(case)   # the reference's own copy, stepped by its own kernels
    mine = ref_bind.RefCudaRun(case)   # a second reference allocation, stepped by this library
    host.initialize()
    mine.initialize()
    host.compute_rhs()
    dq_ref = host.download("dq")
    s = ostc.Solver(case.scheme, case.mech, [_ViewBlock(mine, 0)], case.faces)
    s.initialize()
    s.compute_rhs()
    dq = mine.download("dq")  # written by this library into the reference's array
    o = OracleRun(case)
    o.initialize()
    assert max(rhs_errors(dq, dq_ref, o.flux_scale())) <= 1e-11
    res_r, dt_r = host.rk3_steps(10)
    s.initialize()
    res_g, dt_g = s.rk3_steps(10, history=True)
    assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
    if _reduction_well_defined(case.cells):  # the reference's residual reduction (quirk A19)
        assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    for nm in ("bv", "sv") if case.mech else ("bv",):
        assert max(normwise(mine.download(nm), host.download(nm))) <= 1e-9, nm
    s.close()
