"""The host metric helper (ostc_metric_from_grid, openstc-dev_b200/host/
mesh.cpp) against the reference's own Block::compute_jac_metric
(src/Mesh.cpp:259-521, compiled from the reference sources into
oracle/_ref): bit-identical Jacobians and metric records on warped 3-D grids,
a stretched grid, and a 2-D grid whose k ghost nodes sit at z = k. Runs on the
CPU (both are host code); skipped where the reference build is absent."""
import numpy as np
import pytest

import ostc
import ref_bind

pytestmark = pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")


def _ours(mx, my, mz, ngg, x, y, z):
    b = ostc.HostBlock.allocate(mx, my, mz, ngg, 5, 0)
    ostc.fill_metric(b, np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(z))
    return b.arrays["jac"], b.arrays["metric"]


def _stretched(mx, my, mz, ng, dx):
    """y clustered towards j = 0 (tanh stretching), x and z warped"""
    x, y, z = ostc.grid_coordinates(mx, my, mz, ng, dx, warp=0.05, periodic_k=False)
    j = np.arange(-ng, my + ng, dtype=np.float64)[None, :, None]
    eta = j / (my - 1)
    y = y + dx * (my - 1) * 0.3 * (np.tanh(2 * (eta - 1)) / np.tanh(2.0) + 1 - eta)
    return x, y, z


@pytest.mark.parametrize("dims,ngg,kind", [((12, 9, 7), 2, "warped"), ((10, 8, 6), 3, "warped"),
                                           ((14, 11, 5), 2, "stretched"), ((13, 10, 1), 2, "planar"),
                                           ((9, 12, 1), 3, "planar")])
def test_metric_bit_identical_to_reference(dims, ngg, kind):
    mx, my, mz = dims
    dx = 1e-3
    if kind == "stretched":
        x, y, z = _stretched(mx, my, mz, ngg + 1, dx)
    else:
        x, y, z = ostc.grid_coordinates(mx, my, mz, ngg + 1, dx, warp=0.04, periodic_k=False)
    jac_o, met_o = _ours(mx, my, mz, ngg, x, y, z)
    jac_r, met_r = ref_bind.metric(mx, my, mz, ngg, x, y, z)
    assert np.all(jac_r > 0)
    assert np.array_equal(jac_o.view(np.uint64), jac_r.view(np.uint64))
    assert np.array_equal(met_o["m"].view(np.uint64), met_r["m"].view(np.uint64))

