"""Synthetic meshes written in the reference's input-file formats (grid,
boundary and inner-face files, ostc.write_reference_mesh) for the tests of
the grid pre-processing: a 2-D two-block step like the reference's shipped
grid (a channel block joined to the upper part of a wider block's i-min
face, whose lower part is a second inflow), and a 3-D pair of warped blocks
stacked in j. Coordinates share one smooth warp, so the joined planes
coincide."""
import numpy as np

import ostc


def _warp(x, y, z, L):
    s = 0.02 * L
    return (x + s * np.sin(2 * np.pi * y / L) * np.cos(np.pi * z / L),
            y + s * np.sin(2 * np.pi * x / L),
            z + s * np.sin(np.pi * (x + y) / L))


def step_2d(directory, n=(21, 11, 31, 21), dx=1.0):
    """block 0: n0 x n1 nodes over x in [-(n0-1), 0], y in [n3-n1, n3-1];
    block 1: n2 x n3 nodes over x in [0, n2-1], y in [0, n3-1] (units dx,
    the grid file in mm as the reference's); block 0's i-max plane meets
    block 1's i-min plane over its upper n1 nodes"""
    n0, n1, n2, n3 = n
    L = 40.0 * dx
    coords, dims = [], [(n0, n1, 1), (n2, n3, 1)]
    for (ox, oy, mx, my) in ((-(n0 - 1), n3 - n1, n0, n1), (0, 0, n2, n3)):
        J, I = np.meshgrid(np.arange(my), np.arange(mx), indexing="ij")
        x, y = (I + ox) * dx, (J + oy) * dx
        xw, yw, _ = _warp(x, y, 0 * x, L)
        coords.append((xw[None], yw[None], np.zeros((1, my, mx))))
    bnd = [[(0, n0 - 1, 0, 0, 0, 0, 2), (0, n0 - 1, n1 - 1, n1 - 1, 0, 0, 2), (0, 0, 0, n1 - 1, 0, 0, 5)],
           [(0, n2 - 1, 0, 0, 0, 0, 2), (n2 - 1, n2 - 1, 0, n3 - 1, 0, 0, 6), (0, n2 - 1, n3 - 1, n3 - 1, 0, 0, 2),
            (0, 0, n3 - n1, 0, 0, 0, 9)]]
    inner = [[((n0, n0, 1, n1, 1, 1, 1), (1, 1, n3 - n1 + 1, n3, 1, 1, 2))],
             [((1, 1, n3 - n1 + 1, n3, 1, 1, 2), (n0, n0, 1, n1, 1, 1, 1))]]
    return ostc.write_reference_mesh(directory, dims, coords, bnd, inner)


def stacked_3d(directory, a=(12, 8, 6), b=(12, 7, 6), dx=1.0):
    """block 0 (a) below block 1 (b) in j, aligned axes, shared j plane"""
    L = 20.0 * dx
    coords = []
    for (mx, my, mz), oy in ((a, 0), (b, a[1] - 1)):
        K, J, I = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
        coords.append(_warp(I * dx, (J + oy) * dx, K * dx, L))
    bnd = [[(0, 0, 0, a[1] - 1, 0, a[2] - 1, 5), (a[0] - 1, a[0] - 1, 0, a[1] - 1, 0, a[2] - 1, 6),
            (0, a[0] - 1, 0, 0, 0, a[2] - 1, 2), (0, a[0] - 1, 0, a[1] - 1, 0, 0, 3),
            (0, a[0] - 1, 0, a[1] - 1, a[2] - 1, a[2] - 1, 3)],
           [(0, 0, 0, b[1] - 1, 0, b[2] - 1, 5), (b[0] - 1, b[0] - 1, 0, b[1] - 1, 0, b[2] - 1, 6),
            (0, b[0] - 1, b[1] - 1, b[1] - 1, 0, b[2] - 1, 6), (0, b[0] - 1, 0, b[1] - 1, 0, 0, 3),
            (0, b[0] - 1, 0, b[1] - 1, b[2] - 1, b[2] - 1, 3)]]
    # 3-D inner faces mark the first tangential axis by negative 1-based bounds
    inner = [[((-1, -a[0], a[1], a[1], 1, a[2], 1), (-1, -b[0], 1, 1, 1, b[2], 2))],
             [((-1, -b[0], 1, 1, 1, b[2], 2), (-1, -a[0], a[1], a[1], 1, a[2], 1))]]
    return ostc.write_reference_mesh(directory, [a, b], coords, bnd, inner)
