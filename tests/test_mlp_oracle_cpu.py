"""The numpy restatement of the surrogate network (oracle/mlp_oracle.py)
checked on the CPU: its float64 backpropagation against central finite
differences of its own loss, and the BF16 rounding helper against the
round-to-nearest-even definition."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as M  # noqa: E402


def _params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.normal(0, scale, M.NPARAMS)


def test_parameter_count():
    assert M.NPARAMS == 137482


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    p = _params()
    x = rng.normal(0, 1, (16, M.NIN))
    y = rng.normal(0, 1, (16, M.NOUT))
    g, _ = M.gradients(p, x, y, bf=False)
    idx = rng.choice(M.NPARAMS, 60, replace=False)
    h = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (M.gradients(pp, x, y, bf=False)[1] - M.gradients(pm, x, y, bf=False)[1]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (q, fd, g[q])


def test_bf16_rounding():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 65504.0, 1e-3], dtype=np.float64)
    r = M.bf16(vals)
    # representable in 8 significant bits, nearest to the input
    for v, w in zip(vals, r):
        m, e = np.frexp(w)
        assert m * 256 == np.round(m * 256)
        assert abs(w - v) <= abs(v) * 2 ** -8
    # ties to even: 1 + 2^-8 lies halfway between 1 and 1 + 2^-7
    assert M.bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0
