"""GPU parity of the 2-D path (every block mz == 1): z fluxes skipped, the k
ghost planes copied from k = 0 after the interface exchange of every stage
(eliminate_k_gradient, src/FieldOperation.cuh:372-400, src/RK.cuh:147-153),
the 2-D time step and Roe entropy fix, rho w = 0 in the stage update.
Against the oracle (RHS 1e-11 of the flux scale, histories and states 1e-9),
against the reference's own kernels (oracle/_ref, 2-D Driver sequence),
against this path's own 3-D run of the plane repeated in k, and the tile-table
launches against the per-block ones on a 2-D multi-block SST layout."""
import numpy as np
import pytest

import ostc
from oracle_bind import OracleRun, rhs_errors
from planar_cases import extrude, k_plane, planar_cases, with_fixed_dt

pytestmark = pytest.mark.gpu

NAMES = list(planar_cases())
EQUIVALENT = [n for n in NAMES if n not in ("vortex_muscl_roe", "vortex_aweno", "sst_wall", "sst_h2air_wall")]
DT = {"mixing_h2air": 5e-9, "sst_wall": 1e-8, "sst_h2air_wall": 5e-9}


def _errors(got, ref):
    """normwise per plane, velocity components sharing the largest one's scale"""
    den = [float(np.max(np.abs(ref[l]))) for l in range(ref.shape[0])]
    vel = max(den[1:4]) if ref.shape[0] == 6 else None
    return [float(np.max(np.abs(got[l] - ref[l]))) / ((vel if vel and 1 <= l <= 3 else den[l]) or 1.0)
            for l in range(ref.shape[0])]


def _rhs_errors(got, ref, scale):
    """rhs_errors with the momentum components sharing their largest scale:
    on a 2-D block the rho w flux is rounding noise (Roe's dissipation) or an
    artefact of the characteristic projection (AWENO), not a scale of its own"""
    mom = max(float(np.max(np.abs(ref[l]))) for l in (1, 2, 3))
    sc = np.array(scale, dtype=float)
    sc[1:4] = max(sc[1:4].max(), mom / 1e-2)
    return rhs_errors(got, ref, sc)


def _planar_sst_multiblock():
    return ostc.case_uneven_blocks(layout=ostc.planar_layout((14, 12, 13), (11, 12)), rans_model=2)


@pytest.mark.parametrize("name", NAMES)
def test_planar_rhs_matches_oracle(name):
    case = planar_cases()[name]()
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale(0)
    o.compute_rhs()
    s, blocks = case.solver()
    s.initialize()
    s.compute_rhs()
    err = _rhs_errors(blocks[0].download("dq"), o.blocks[0].arrays["dq"], scale)
    assert max(err) <= 1e-11, err
    s.close()


@pytest.mark.parametrize("name", NAMES)
def test_planar_history_matches_oracle(name):
    """5 RK3 steps at the CFL dt: dt, residuals and states to 1e-9; w stays
    exactly 0 and every k ghost plane is a copy of k = 0"""
    case = planar_cases()[name]()
    n = 5
    o = OracleRun(case)
    o.initialize()
    res_o, dt_o = o.rk3_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    ng = case.blocks[0].ngg
    for arr in ("bv", "sv"):
        got = blocks[0].download(arr)
        if not got.size:
            continue
        assert max(_errors(got, o.blocks[0].arrays[arr])) <= 1e-9, arr
        for k in range(-ng, ng + 1):
            assert np.array_equal(k_plane(got, ng, k), k_plane(got, ng)), (arr, k)
    assert not np.any(blocks[0].download("bv")[3])
    s.close()


@pytest.mark.parametrize("name", EQUIVALENT)
def test_planar_equals_extruded(name):
    """the 2-D run and this path's 3-D run of the same plane repeated 4 times
    in k (unit k spacing, periodic k faces) at a fixed dt agree to round-off
    on every k plane (schemes without a dimension-dependent term)"""
    base = planar_cases()[name]()
    dt = DT.get(name, 1e-7)
    out = []
    for c in (with_fixed_dt(base, dt), extrude(base, 4, dt)):
        s, blocks = c.solver()
        s.initialize()
        s.rk3_steps(3)
        out.append((blocks[0].download("bv"), blocks[0].download("sv")))
        s.close()
    ng = base.blocks[0].ngg
    for a2, a3 in zip(out[0], out[1]):
        if not a2.size:
            continue
        ref = k_plane(a2, ng)
        for k in range(4):
            got = k_plane(a3, ng, k)
            for l in range(ref.shape[0]):
                den = np.max(np.abs(ref[l])) or 1.0
                assert np.max(np.abs(got[l] - ref[l])) <= 1e-13 * den, (k, l)


def test_planar_multiblock_batched_and_oracle():
    """six 2-D SST blocks joined by interfaces: the tile-table launches equal
    the per-block launches bitwise, and both follow the oracle (fixed dt)"""
    case = with_fixed_dt(_planar_sst_multiblock(), 1e-8)
    n = 4
    o = OracleRun(case)
    o.initialize()
    o.rk3_steps(n)
    out = {}
    for batched in (True, False):
        s, blocks = case.solver()
        s.set_batching(batched)
        s.initialize()
        s.rk3_steps(n)
        out[batched] = [(b.download("bv"), b.download("sv"), b.download("mut")) for b in blocks]
        s.close()
    for x, y in zip(out[True], out[False]):
        for a, b in zip(x, y):
            assert np.array_equal(a, b)
    for b, (bv, sv, mut) in enumerate(out[True]):
        assert max(_errors(bv, o.blocks[b].arrays["bv"])) <= 1e-9, b
        assert max(_errors(sv, o.blocks[b].arrays["sv"])) <= 1e-9, b
        ref = o.blocks[b].arrays["mut"]
        assert np.max(np.abs(mut - ref)) <= 1e-9 * np.max(np.abs(ref)), b


def _reference_case(name):
    case = planar_cases()[name]()
    for f in case.faces:  # the reference's air + SST far field reads unset scalars (A20)
        if case.scheme.rans_model == 2 and f.type_label == ostc.BC_FARFIELD:
            f.type_label = ostc.BC_OUTFLOW
    return case


@pytest.mark.skipif(not __import__("ref_bind").available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", NAMES)
def test_planar_matches_reference_build(name):
    """the reference's own kernels in its 2-D sequence (eliminate_k_gradient,
    no z fluxes, 16 x 16 x 1 launches, param->dim = 2): one RHS (1e-11) and
    5 RK3 steps at the CFL dt (dt, residuals and states to 1e-9)"""
    import ref_bind

    case = _reference_case(name)
    o = OracleRun(case)
    o.initialize()
    scale = o.flux_scale(0)
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    r.compute_rhs()
    s, blocks = case.solver()
    s.initialize()
    s.compute_rhs()
    assert max(_rhs_errors(blocks[0].download("dq"), r.download("dq"), scale)) <= 1e-11
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
    for arr in ("bv", "sv"):
        got = blocks2[0].download(arr)
        if got.size:
            assert max(_errors(got, r2.download(arr))) <= 1e-9, arr
    s2.close()


@pytest.mark.parametrize("name,implicit_method", [("wall_farfield", 0), ("wall_farfield", 1), ("sst_wall", 0),
                                                  ("sst_wall", 1), ("mixing_h2air", 1), ("sst_h2air_wall", 1)])
def test_planar_steady(name, implicit_method):
    """the steady path on 2-D blocks (SteadySim.cuh:51-126 with its
    eliminate_k_gradient, DPLUR without k neighbours): 4 iterations against
    the oracle (residuals and states 1e-9) and the reference's kernels"""
    import ref_bind

    case = ostc.make_steady(_reference_case(name), implicit_method=implicit_method, dplur_inner_step=2)
    n = 4
    o = OracleRun(case)
    o.initialize()
    res_o = o.steady_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g = s.steady_steps(n, history=True)
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for arr in ("bv", "sv"):
        got = blocks[0].download(arr)
        if got.size:
            assert max(_errors(got, o.blocks[0].arrays[arr])) <= 1e-9, arr
    s.close()
    if not ref_bind.available():
        return
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    res_r = r.steady_steps(n)
    s2, blocks2 = case.solver()
    s2.initialize()
    s2.steady_steps(n)
    for arr in ("bv", "sv"):
        got = blocks2[0].download(arr)
        if got.size:
            assert max(_errors(got, r.download(arr))) <= 1e-9, arr
    if res_r is not None:
        assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    s2.close()
