"""CPU restatement (numpy) of the chemistry surrogate's network and of its
gradients: the checker of the training kernels in openstc-dev_b200/csrc/
mlp.cu. TEST INFRASTRUCTURE ONLY: tests/ may import it; the product never
does.

The network is a 12-256-256-256-10 perceptron with SiLU activations. With
bf16=True the restatement rounds exactly where the GPU path stores BF16
(the packed inputs, the weights, the SiLU activations and the output
gradients that feed the tensor-core products) and computes everything else
in float64, so the GPU gradients differ from it only by FP32 accumulation
order (and the rare BF16 rounding flip that order causes). With bf16=False
it is plain float64 backpropagation, checked against finite differences.

No reference counterpart: the reference has no learned chemistry."""
import numpy as np

NIN, NH, NOUT = 12, 256, 10
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(flat):
    out, q = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(flat[q:q + n], dtype=np.float64).reshape(shp)
        q += n
    return out


def flatten(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(a):
    """round to the nearest BF16 (ties to even) through float32"""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, bf=True):
    """x [n][12] standardised -> (outputs [n][10], cache)"""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    p = unflatten(params) if not isinstance(params, dict) else params
    a0 = r(x)
    W = [r(p["W1"]), r(p["W2"]), r(p["W3"]), r(p["W4"])]
    b = [p["b1"], p["b2"], p["b3"], p["b4"]]
    acts, zs = [a0], []
    h = a0
    for layer in range(4):
        z = h @ W[layer].T + b[layer]
        zs.append(z)
        if layer < 3:
            h = r(silu(z))
            acts.append(h)
    return zs[3], (acts, zs, W)


def gradients(params, x, y, bf=True):
    """mean squared error over n rows and 10 outputs; returns (flat grads, loss)"""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    out, (acts, zs, W) = forward(params, x, bf)
    n = x.shape[0]
    diff = out - y
    loss = float(np.mean(diff * diff))
    dz = 2.0 * diff / (n * NOUT)
    g = {}
    names = [("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4")]
    for layer in range(3, -1, -1):
        dzb = r(dz)
        g[names[layer][0]] = dzb.T @ acts[layer]
        g[names[layer][1]] = dz.sum(axis=0)
        if layer == 0:
            break
        da = dzb @ W[layer]
        dz = da * dsilu(zs[layer - 1])
    return flatten(g), loss
