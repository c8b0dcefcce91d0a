"""Building the chemistry surrogate: training data from the FP64
point-implicit integrator, feature / target scaling, the training loop on
the library's own kernels (ostc.Surrogate.train_step), and its evaluation.

Inputs of the network (12): log T, log p, log(max(Y_k, 0) + 1e-10) for the nine
species, log dt. Outputs (10): the integrator's rates r = dY_k / dt and
dT / dt (increments vary over the two decades of dt mostly through the dt
factor, which the rates remove), learned as z = asinh(r / r0) with r0 a
thousandth of the rate's standard deviation: small rates keep relative
precision (a radical's formation enthalpy turns a 1e-6 error in its mass
fraction into a kelvin of temperature), large ones are compressed
logarithmically. Features and z are standardised with the training set's mean and standard deviation; the
envelope (per-feature min / max of the training inputs, widened on each side
by ENVELOPE_MARGIN of the feature's range) bounds where the network is
trusted. The formula of the features is the one of csrc/surrogate.cuh:
surrogate_features.

Training states (the chemistry-surrogate configuration: "states sampled from
runs of" the reacting mixing layer) come from trajectory_states: snapshots of
FP64 operator-split runs of the layer (chem_mode 1), next to the seeded
synthetic states of ostc.sample_chem_states that cover the wider envelope
(T 300-3000 K, p 0.5-3 atm, dt 1e-9..1e-7 s).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

import ostc

ATOMIC_MASS = {"H": 1.008, "O": 15.999, "N": 14.007, "C": 12.011, "AR": 39.95, "Ar": 39.95, "HE": 4.0026}


def features(T, p, Y, dt):
    """[n][12] float64 features (numpy or torch, species-major Y [9][n])"""
    try:
        import torch

        if isinstance(T, torch.Tensor):
            return torch.stack([torch.log(T), torch.log(p)] +
                               [torch.log(Y[l].clamp_min(0) + 1e-10) for l in range(Y.shape[0])] + [torch.log(dt)],
                               dim=1)
    except ImportError:  # pragma: no cover
        pass
    return np.stack([np.log(T), np.log(p)] + [np.log(np.maximum(Y[l], 0) + 1e-10) for l in range(Y.shape[0])] +
                    [np.log(dt)], axis=1)


@dataclass
class Dataset:
    F: "object"   # [n][12] float64 raw features (torch, cuda)
    G: "object"   # [n][10] float64 raw targets: dY_k / dt, dT / dt (torch, cuda)
    T: "object"
    p: "object"
    Y: "object"
    dt: "object"


def label_states(solver: "ostc.Solver", T, p, Y, dt, chunk: int = 1 << 21) -> Dataset:
    """Runs the FP64 integrator on the states (numpy) and keeps the converged ones."""
    import torch

    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (T, p, Y, dt)]
    Tt, pt, Yt, dtt = dev
    n = Tt.numel()
    dY = torch.empty_like(Yt)
    dT = torch.empty_like(Tt)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        sub = [Tt[a:b].contiguous(), pt[a:b].contiguous(), Yt[:, a:b].contiguous(), dtt[a:b].contiguous()]
        d1, d2 = solver.chem_point_implicit(*sub)
        dY[:, a:b] = d1
        dT[a:b] = d2
    ok = torch.isfinite(dT)
    F = features(Tt, pt, Yt, dtt)[ok]
    G = (torch.cat([dY.T, dT[:, None]], dim=1) / dtt[:, None])[ok]
    return Dataset(F, G, Tt[ok], pt[ok], Yt[:, ok], dtt[ok])


@dataclass
class Scaling:
    in_mean: np.ndarray
    in_std: np.ndarray
    out_mean: np.ndarray
    out_std: np.ndarray
    in_min: np.ndarray
    in_max: np.ndarray
    out_r0: np.ndarray


R0_FRACTION = 1e-3
# the trusted envelope reaches this fraction of each feature's training range
# beyond its training minimum and maximum: a flow step moves states a little
# past the extremes of the data (the cold stream cools below its 300 K inflow
# by expansion), where the network is still accurate
ENVELOPE_MARGIN = 0.02


def _transform(G, r0):
    import torch

    return torch.asinh(G / r0)


def fit_scaling(d: Dataset) -> Scaling:
    import torch

    F = d.F.double()
    G = d.G.double()
    r0 = (R0_FRACTION * G.std(0)).clamp_min(1e-30)
    Z = _transform(G, r0)
    fm, fs = F.mean(0), F.std(0).clamp_min(1e-12)
    gm, gs = Z.mean(0), Z.std(0).clamp_min(1e-12)
    lo, hi = F.min(0).values, F.max(0).values
    pad = ENVELOPE_MARGIN * (hi - lo)
    return Scaling(fm.cpu().numpy(), fs.cpu().numpy(), gm.cpu().numpy(), gs.cpu().numpy(),
                   (lo - pad).cpu().numpy(), (hi + pad).cpu().numpy(), r0.cpu().numpy())


def standardise(d: Dataset, sc: Scaling):
    import torch

    dev = d.F.device
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    X = ((d.F - t(sc.in_mean)) / t(sc.in_std)).float().contiguous()
    Yt = ((_transform(d.G, t(sc.out_r0)) - t(sc.out_mean)) / t(sc.out_std)).float().contiguous()
    return X, Yt


@dataclass
class TrainLog:
    steps: int = 0
    seconds: float = 0.0
    loss: List[float] = field(default_factory=list)


def train(sur: "ostc.Surrogate", X, Yt, epochs: int = 20, batch: int = 65536, lr: float = 1e-3, seed: int = 0,
          log_every: int = 50) -> TrainLog:
    """Adam with cosine learning-rate decay over epochs x (n / batch) steps;
    batches are drawn from a seeded permutation each epoch."""
    import torch

    n = X.shape[0]
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    loss = torch.zeros(1, dtype=torch.float32, device=X.device)
    log = TrainLog()
    torch.cuda.synchronize()
    t0 = time.time()
    step = 0
    for _ in range(epochs):
        perm = torch.randperm(n, device=X.device, generator=g)
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            xb, yb = X[idx].contiguous(), Yt[idx].contiguous()
            lr_t = 0.5 * lr * (1 + math.cos(math.pi * step / total))
            sur.train_step(xb, yb, lr_t, loss)
            if step % log_every == 0 or step == total - 1:
                log.loss.append(float(loss.item()) / (xb.shape[0] * ostc.SURR_OUT))
            step += 1
    torch.cuda.synchronize()
    log.steps = step
    log.seconds = time.time() - t0
    return log


def trajectory_states(n: int, size=(64, 256, 64), seeds=(5, 6), steps: int = 40, every: int = 10, seed: int = 0,
                      dt_range=(1e-9, 1e-7)):
    """n cell states (T, p, Y [n_spec][n], dt as numpy arrays) sampled from
    snapshots of FP64 operator-split runs of the reacting mixing layer
    (chem_mode 1, one run per noise seed, a snapshot every `every` of
    `steps` RK3 steps); dt log-uniform in dt_range, as the labeller's
    increments are learned over that span."""
    import torch

    snaps = []
    for sd in seeds:
        c = ostc.case_mixing_layer(*size, seed=sd)
        c.scheme.chem_mode = 1
        s, blocks = c.solver()
        s.initialize()
        g = c.blocks[0].ngg
        for _ in range(0, steps, every):
            s.rk3_steps(every)
            bv, sv = blocks[0].t["bv"], blocks[0].t["sv"]
            snaps.append((bv[5, g:-g, g:-g, g:-g].reshape(-1), bv[4, g:-g, g:-g, g:-g].reshape(-1),
                          sv[:, g:-g, g:-g, g:-g].reshape(sv.shape[0], -1)))
        torch.cuda.synchronize()
        s.close()
        del blocks
    T = torch.cat([x[0] for x in snaps])
    p = torch.cat([x[1] for x in snaps])
    Y = torch.cat([x[2] for x in snaps], dim=1)
    rng = np.random.default_rng(seed)
    pick = torch.from_numpy(rng.choice(T.numel(), min(n, T.numel()), replace=False)).to(T.device)
    dt = 10 ** rng.uniform(np.log10(dt_range[0]), np.log10(dt_range[1]), pick.numel())
    return (T[pick].cpu().numpy(), p[pick].cpu().numpy(), np.ascontiguousarray(Y[:, pick].cpu().numpy()), dt)


def set_checks(sur: "ostc.Surrogate", mech: "ostc.Mechanism", tol_elem: float = 1e-4, tol_T: float = 1.0):
    els = ostc.species_elements(mech.names)
    names = sorted(els)
    counts = np.stack([els[e] for e in names])
    mass = np.array([ATOMIC_MASS[e] for e in names])
    sur.set_checks(counts, mass, tol_elem, tol_T)


def build(solver: "ostc.Solver", mech: "ostc.Mechanism", n_train: int = 4_000_000, epochs: int = 20,
          batch: int = 65536, lr: float = 1e-3, seed: int = 1, extra_states=None):
    """The whole pipeline: sample states (ostc.sample_chem_states, plus any
    extra (T, p, Y, dt) arrays, e.g. cells of a flow run), label them with the
    FP64 integrator, fit the scaling, train. Returns (surrogate, scaling, log)."""
    T, p, Y, dt = ostc.sample_chem_states(mech, n_train, seed=seed)
    if extra_states is not None:
        T = np.concatenate([T, extra_states[0]])
        p = np.concatenate([p, extra_states[1]])
        Y = np.concatenate([Y, extra_states[2]], axis=1)
        dt = np.concatenate([dt, extra_states[3]])
    d = label_states(solver, T, p, Y, dt)
    sc = fit_scaling(d)
    X, Yt = standardise(d, sc)
    sur = ostc.Surrogate(max_batch=batch, seed=seed)
    sur.set_scaling(sc.in_mean, sc.in_std, sc.out_mean, sc.out_std, sc.in_min, sc.in_max, sc.out_r0)
    set_checks(sur, mech)
    log = train(sur, X, Yt, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return sur, sc, log


def errors(solver, sur, T, p, Y, dt):
    """Surrogate chemistry step vs the FP64 integrator on the same states
    (torch cuda tensors): per-state |dT| and max_k |dY_k| errors, the
    fallback count, and the rejected mask."""
    import torch

    dY_s, dT_s, nfb = solver.chem_surrogate(sur, T, p, Y, dt)
    dY_r, dT_r = solver.chem_point_implicit(T, p, Y, dt)
    eT = (dT_s - dT_r).abs()
    eY = (dY_s - dY_r).abs().max(dim=0).values
    return eT, eY, nfb


def save(path, sur: "ostc.Surrogate", sc: Scaling):
    np.savez(path, params=sur.params(), in_mean=sc.in_mean, in_std=sc.in_std, out_mean=sc.out_mean,
             out_std=sc.out_std, in_min=sc.in_min, in_max=sc.in_max, out_r0=sc.out_r0)


def load(path, mech: "ostc.Mechanism", max_batch: int = 65536):
    z = np.load(path)
    sc = Scaling(z["in_mean"], z["in_std"], z["out_mean"], z["out_std"], z["in_min"], z["in_max"], z["out_r0"])
    sur = ostc.Surrogate(max_batch=max_batch)
    sur.set_params(z["params"])
    sur.set_scaling(sc.in_mean, sc.in_std, sc.out_mean, sc.out_std, sc.in_min, sc.in_max, sc.out_r0)
    set_checks(sur, mech)
    return sur, sc


def main(argv=None):
    """Train a surrogate on the 9-species H2-air mechanism and evaluate it on
    held-out states against the FP64 integrator:
        python openstc-dev_b200/surrogate.py --train 4000000 --epochs 20 --eval 1000000 [--save f.npz]"""
    import argparse

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--eval", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--save", default=None)
    a = ap.parse_args(argv)
    case = ostc.case_premixed_box(8, 8, 4)
    solver, _ = case.solver()
    sur, sc, log = build(solver, case.mech, n_train=a.train, epochs=a.epochs, seed=a.seed)
    T, p, Y, dt = [torch.from_numpy(x).cuda() for x in ostc.sample_chem_states(case.mech, a.eval, seed=a.seed + 1000)]
    eT, eY, nfb = errors(solver, sur, T, p, Y, dt)
    print({"train_states": a.train, "epochs": a.epochs, "train_s": round(log.seconds, 2), "final_loss": log.loss[-1],
           "eval_states": a.eval, "fallback_fraction": nfb / a.eval, "max_dT_err_K": float(eT.max()),
           "p99_dT_err_K": float(eT.quantile(0.99)), "max_dY_err": float(eY.max()),
           "p99_dY_err": float(eY.quantile(0.99))})
    if a.save:
        save(a.save, sur, sc)


if __name__ == "__main__":
    main()
