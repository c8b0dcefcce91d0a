"""GPU checks of the surrogate network's hand-written training kernels
(csrc/mlp.cu) against the numpy restatement (oracle/mlp_oracle.py), which
rounds to BF16 exactly where the GPU path stores BF16: the forward outputs
and every parameter gradient agree to FP32-accumulation-order differences
(bar 2e-3 relative to each tensor's largest entry), and Adam steps reduce
the loss on a learnable target."""
import sys
from pathlib import Path

import numpy as np
import pytest

import ostc

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, M.NIN)).astype(np.float32)
    y = rng.normal(0, 1, (n, M.NOUT)).astype(np.float32)
    return x, y


def _per_tensor_err(a, b):
    out, q = {}, 0
    for name, shp in M.SHAPES:
        n = int(np.prod(shp))
        den = max(np.max(np.abs(b[q:q + n])), 1e-30)
        out[name] = float(np.max(np.abs(a[q:q + n] - b[q:q + n])) / den)
        q += n
    return out


@pytest.mark.parametrize("n", [700, 8192])
def test_forward_and_gradients_match_oracle(n):
    import torch

    s = ostc.Surrogate(max_batch=8192, seed=3)
    p = s.params().astype(np.float64)
    x, y = _data(n, 4)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    out = s.forward(xt).cpu().numpy()
    ref, _ = M.forward(p, x.astype(np.float64))
    assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) <= 2e-3
    g, loss = s.gradients(xt, yt)
    gref, lref = M.gradients(p, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - lref) <= 1e-3 * lref
    err = _per_tensor_err(g.astype(np.float64), gref)
    assert max(err.values()) <= 2e-3, err
    s.close()


@pytest.mark.parametrize("n", [1, 127, 128, 5000, 300000])
def test_tensor_core_forward_matches(n):
    """The tcgen05 inference kernel (TMEM accumulators, 128-row tiles, ragged
    last tile) against the mma.sync forward and the BF16-emulating oracle."""
    import torch

    s = ostc.Surrogate(max_batch=max(n, 8), seed=11)
    p = s.params().astype(np.float64)
    # trained-like scale: random weights with a spread of magnitudes
    rng = np.random.default_rng(n)
    s.set_params((p * rng.uniform(0.5, 2.0, p.size)).astype(np.float32))
    p = s.params().astype(np.float64)
    x, _ = _data(n, 9)
    xt = torch.from_numpy(x).cuda()
    y_tc = s.forward_tc(xt).cpu().numpy()
    y_mma = s.forward(xt).cpu().numpy() if n <= s.max_batch else None
    ref, _ = M.forward(p, x.astype(np.float64))
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(y_tc - ref)) / scale <= 2e-3
    if y_mma is not None:
        assert np.max(np.abs(y_tc - y_mma)) / scale <= 2e-3
    s.close()


def test_adam_reduces_loss():
    import torch

    rng = np.random.default_rng(7)
    n = 4096
    x = rng.normal(0, 1, (n, M.NIN)).astype(np.float32)
    w = rng.normal(0, 0.5, (M.NIN, M.NOUT))
    y = np.tanh(x @ w).astype(np.float32)  # a smooth learnable map
    s = ostc.Surrogate(max_batch=n, seed=5)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    _, l0 = s.gradients(xt, yt)
    for _ in range(200):
        s.train_step(xt, yt, 1e-3)
    _, l1 = s.gradients(xt, yt)
    assert l1 < 0.05 * l0, (l0, l1)
    s.close()
