"""The CPU oracle pinned against golden vectors produced by the reference
itself: its own CUDA kernels, compiled from the reference sources and run on
a B200 by tests/golden/make_golden.py, on small seeded cases covering every
inviscid scheme, the boundary conditions, block interfaces, the steady path
with EPI / DA / DPLUR, k-omega SST with air and with the H2-air mixture, and
2-D blocks. No GPU is needed here.

Bars: 1e-11 on one RHS evaluation (conditioning-aware, rhs_errors), 1e-9
normwise on interior states and on residual / dt histories after the steps
(the host libm differs from CUDA's in the last ulp, which the nonlinear
updates amplify)."""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

from oracle_bind import OracleRun, normwise, rhs_errors

GOLDEN = Path(__file__).resolve().parent / "golden"
_spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

FILES = sorted(GOLDEN.glob("*.npz"))


def test_golden_vectors_present():
    assert {f.stem for f in FILES} == set(make_golden.CASES), "regenerate with tests/golden/make_golden.py"


@pytest.mark.parametrize("path", FILES, ids=[f.stem for f in FILES])
def test_oracle_matches_reference_golden(path):
    gold = np.load(path)
    build, mode, steps = make_golden.CASES[path.stem]
    case = build()
    for b, blk in enumerate(case.blocks):
        assert str(gold["digest_%d" % b]) == make_golden.input_digest(blk), "case builder changed"
    o = OracleRun(case)
    o.initialize()
    for b, blk in enumerate(case.blocks):
        scale = o.flux_scale(b)
        scale[1:4] = scale[1:4].max()  # momentum components share a scale (rho w is rounding noise in 2-D)
        dq = make_golden.interior(o.blocks[b].arrays["dq"], blk.dq_ngg)
        err = rhs_errors(dq, gold["dq_%d" % b], scale)
        assert max(err) <= 1e-11, (b, err)
    o2 = OracleRun(case)
    o2.initialize()
    if mode == "rk3":
        res, dts = o2.rk3_steps(int(steps))
        if bool(gold["reduction_ok"]):
            assert np.max(np.abs(dts - gold["dt"]) / gold["dt"]) <= 1e-9
    else:
        res = o2.steady_steps(int(steps))
    if bool(gold["reduction_ok"]):
        assert np.max(np.abs(res - gold["res"]) / gold["res"]) <= 1e-9
    for b, blk in enumerate(case.blocks):
        got = make_golden.interior(o2.blocks[b].arrays["bv"], blk.ngg)
        err = normwise(got, gold["bv_%d" % b])
        vel = max(float(np.max(np.abs(gold["bv_%d" % b][l]))) for l in (1, 2, 3))
        for l in (1, 2, 3):  # velocity components share the largest one's scale
            err[l] = float(np.max(np.abs(got[l] - gold["bv_%d" % b][l]))) / vel
        assert max(err) <= 1e-9, (b, err)
        if blk.n_spec + blk.n_turb:
            got = make_golden.interior(o2.blocks[b].arrays["sv"], blk.ngg)
            assert max(normwise(got, gold["sv_%d" % b])) <= 1e-9, b
