"""GPU parity of the multi-block path: six blocks of uneven sizes joined by
fourteen 1-to-1 interfaces (inner_communication, src/DataCommunication.cuh:
58-110), against the CPU oracle and against the reference's own CUDA
kernels driving the same blocks (oracle/_ref/libostc_ref_cuda.so).

Block sizes are (17, 15, 12) x (14, 17) x 10 cells: every block keeps the
reference's block reductions (dt minimum, residual sums) well defined, so
its time steps and residuals can be compared too. Bars as for one block:
1e-11 per RHS evaluation (conditioning-aware, oracle_bind.rhs_errors),
1e-9 on states, dt and residuals after 10 steps."""
import numpy as np
import pytest

import ostc
import ref_bind
from oracle_bind import OracleRun, normwise, rhs_errors

pytestmark = pytest.mark.gpu

NX, NY, MZ = (17, 15, 12), (14, 17), 10
SCHEMES = {"aweno": (4, 2), "roe_muscl": (2, 2), "ausm_muscl": (2, 3), "hllc_nnd2": (3, 4)}


def _case(name):
    recon, inv = SCHEMES[name]
    return ostc.case_multiblock(NX, NY, MZ, reconstruction=recon, inviscid_scheme=inv)


def _reduction_well_defined(cells):
    # see test_parity_refcuda_gpu._reduction_well_defined
    nb = (cells + 127) // 128
    v1, v2 = cells - (nb - 1) * 128, nb
    return all(v == 128 or v % 32 for v in (v1, v2))


@pytest.mark.parametrize("name", list(SCHEMES))
def test_multiblock_rhs_matches_oracle(name):
    case = _case(name)
    o = OracleRun(case)
    o.initialize()
    scales = [o.flux_scale(b) for b in range(len(case.blocks))]
    o.compute_rhs()
    s, blocks = case.solver()
    s.initialize()
    s.compute_rhs()
    for b in range(len(blocks)):
        err = rhs_errors(blocks[b].download("dq"), o.blocks[b].arrays["dq"], scales[b])
        assert max(err) <= 1e-11, (b, err)
        for arr in ("bv", "cv"):
            assert max(normwise(blocks[b].download(arr), o.blocks[b].arrays[arr])) <= 1e-14, (b, arr)


@pytest.mark.parametrize("name", ["aweno", "roe_muscl"])
def test_multiblock_history_matches_oracle(name):
    case = _case(name)
    n = 10
    o = OracleRun(case)
    o.initialize()
    res_o, dt_o = o.rk3_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for b in range(len(blocks)):
        err = normwise(blocks[b].download("bv"), o.blocks[b].arrays["bv"])
        assert max(err) <= 1e-9, (b, err)


def test_multiblock_split_equals_whole_grid_on_gpu():
    """Decomposition invariance of one RHS on the GPU path (MUSCL + Roe):
    the split grid reproduces the unsplit grid's dq block by block."""
    mb = _case("roe_muscl")
    sb = ostc.case_multiblock((sum(NX) - len(NX) + 1,), (sum(NY) - len(NY) + 1,), MZ, reconstruction=2,
                              inviscid_scheme=2)
    s1, b1 = mb.solver()
    s1.initialize()
    s1.compute_rhs()
    s2, b2 = sb.solver()
    s2.initialize()
    s2.compute_rhs()
    whole = b2[0].download("dq")
    scale = np.max(np.abs(whole), axis=(1, 2, 3))
    ox = np.cumsum([0] + [m - 1 for m in NX])
    oy = np.cumsum([0] + [m - 1 for m in NY])
    q = 0
    for bj, my in enumerate(NY):
        for bi, mx in enumerate(NX):
            got = b1[q].download("dq")
            sub = whole[:, :, oy[bj]:oy[bj] + my, ox[bi]:ox[bi] + mx]
            err = np.max(np.abs(got - sub), axis=(1, 2, 3)) / scale
            assert np.all(err <= 1e-13), (q, err)
            q += 1


@pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", ["aweno", "roe_muscl"])
def test_multiblock_matches_reference_build(name):
    case = _case(name)
    assert all(_reduction_well_defined(b.mx * b.my * b.mz) for b in case.blocks)
    r = ref_bind.RefCudaRun(case)
    r.initialize()
    r.compute_rhs()
    o = OracleRun(case)
    o.initialize()
    scales = [o.flux_scale(b) for b in range(len(case.blocks))]
    s, blocks = case.solver()
    s.initialize()
    s.compute_rhs()
    for b in range(len(blocks)):
        dq_ref = r.download("dq", b)
        assert max(rhs_errors(blocks[b].download("dq"), dq_ref, scales[b])) <= 1e-11, b
    n = 10
    r2 = ref_bind.RefCudaRun(case)
    r2.initialize()
    res_r, dt_r = r2.rk3_steps(n)
    s2, blocks2 = case.solver()
    s2.initialize()
    res_g, dt_g = s2.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
    assert np.max(np.abs(res_g - res_r) / res_r) <= 1e-9
    for b in range(len(blocks2)):
        err = normwise(blocks2[b].download("bv"), r2.download("bv", b))
        assert max(err) <= 1e-9, (b, err)
