"""Metric and Jacobian of a structured block from its node coordinates, in
numpy: a restatement of cfd::Block::compute_jac_metric (src/Mesh.cpp:259-521)
for the CPU legs. Test and measurement infrastructure: used by tests/ and by
bench.py's CPU baseline / reference arm (which must not load the product
library) to build the synthetic workloads' geometry, never by the product path.

Coordinates carry ngg+1 ghost layers; outputs carry ngg. Second-order central
differences of x, y, z along (xi, eta, zeta) at every point of [-ngg, m+ngg),
J = det d(x,y,z)/d(xi,eta,zeta), metric row d = the cofactor row / J
(Mesh.cpp:270-300). A non-positive interior J is an error (Mesh.cpp:282-288);
in the ghost slabs such a point takes the values of its neighbour towards the
block (Mesh.cpp:321-326 and the following slabs), applied layer by layer from
the inside out. The same formulas in the same association order as the
reference, so the result is bit-identical to it.
"""
import numpy as np

METRIC_DTYPE = np.dtype([("bias", "<i4"), ("pad", "<i4"), ("m", "<f8", (9,))])


def metric(mx, my, mz, ngg, x, y, z):
    """(jac, metric) as ghosted arrays of shape (mz+2g, my+2g, mx+2g),
    metric in METRIC_DTYPE (80-byte gxl::Matrix<real,3,3,1> records)."""
    x, y, z = (np.asarray(a, dtype=np.float64) for a in (x, y, z))
    g = ngg

    def d(a, axis):
        # central difference over [-g, m+g) of an array with g+1 ghost layers
        sl_p = [slice(1, -1)] * 3
        sl_m = [slice(1, -1)] * 3
        sl_p[axis] = slice(2, None)
        sl_m[axis] = slice(0, -2)
        return (a[tuple(sl_p)] - a[tuple(sl_m)]) * 0.5

    # numpy axes are (k, j, i): xi = axis 2, eta = axis 1, zeta = axis 0
    dxd1, dyd1, dzd1 = d(x, 2), d(y, 2), d(z, 2)
    dxd2, dyd2, dzd2 = d(x, 1), d(y, 1), d(z, 1)
    dxd3, dyd3, dzd3 = d(x, 0), d(y, 0), d(z, 0)
    jac = (dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 - dxd2 * dyd1 * dzd3 -
           dxd3 * dyd2 * dzd1)
    m = np.empty(jac.shape + (9,))
    m[..., 0] = (dyd2 * dzd3 - dyd3 * dzd2) / jac
    m[..., 1] = (dxd3 * dzd2 - dxd2 * dzd3) / jac
    m[..., 2] = (dxd2 * dyd3 - dxd3 * dyd2) / jac
    m[..., 3] = (dyd3 * dzd1 - dyd1 * dzd3) / jac
    m[..., 4] = (dxd1 * dzd3 - dxd3 * dzd1) / jac
    m[..., 5] = (dxd3 * dyd1 - dxd1 * dyd3) / jac
    m[..., 6] = (dyd1 * dzd2 - dyd2 * dzd1) / jac
    m[..., 7] = (dxd2 * dzd1 - dxd1 * dzd2) / jac
    m[..., 8] = (dxd1 * dyd2 - dxd2 * dyd1) / jac
    interior = jac[g:g + mz, g:g + my, g:g + mx]
    if not np.all(interior > 0):
        raise ValueError("non-positive Jacobian inside the block")
    # ghost points with a non-positive Jacobian copy their inward neighbour
    K, J, I = np.meshgrid(np.arange(-g, mz + g), np.arange(-g, my + g), np.arange(-g, mx + g), indexing="ij")
    di = np.where(I < 0, -I, np.where(I >= mx, I - mx + 1, 0))
    dj = np.where(J < 0, -J, np.where(J >= my, J - my + 1, 0))
    dk = np.where(K < 0, -K, np.where(K >= mz, K - mz + 1, 0))
    layer = np.maximum(di, np.maximum(dj, dk))
    for lay in range(1, g + 1):
        bad = (layer == lay) & ~(jac > 0)
        if not np.any(bad):
            continue
        kk, jj, ii = np.nonzero(bad)
        ki, ji, ii_ = K[bad], J[bad], I[bad]
        ni = np.where(ii_ < 0, ii_ + 1, np.where(ii_ >= mx, ii_ - 1, ii_)) + g
        nj = np.where(ji < 0, ji + 1, np.where(ji >= my, ji - 1, ji)) + g
        nk = np.where(ki < 0, ki + 1, np.where(ki >= mz, ki - 1, ki)) + g
        jac[kk, jj, ii] = jac[nk, nj, ni]
        m[kk, jj, ii] = m[nk, nj, ni]
    met = np.zeros(jac.shape, dtype=METRIC_DTYPE)
    met["bias"] = 4  # gxl::Matrix<real,3,3,1>::bias_ = 1*(3+1)
    met["m"] = m
    return jac, met
