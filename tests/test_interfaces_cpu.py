"""Block-to-block interfaces in the oracle (CPU): the 1-to-1 exchange of
inner_communication (src/DataCommunication.cuh:58-110) checked through a
property that needs no reference run. A grid split into blocks that share
their face planes, initialised from one global field, must give the same
right-hand side as the unsplit grid wherever the scheme's stencils stay
local: each block's ghost layers hold its neighbour's interior, and the
shared plane is computed from identical stencils in both blocks.

The AWENO path is exempt: its central correction covers only the first
n - 2 ngg points of each line (quirk A4), so its RHS depends on where the
blocks end, in the reference as well."""
import numpy as np
import pytest

import ostc
from oracle_bind import OracleRun

NX, NY, MZ = (17, 15, 12), (14, 17), 6


def _split_vs_whole(reconstruction, inviscid_scheme):
    mb = ostc.case_multiblock(NX, NY, MZ, reconstruction=reconstruction, inviscid_scheme=inviscid_scheme)
    sb = ostc.case_multiblock((sum(NX) - len(NX) + 1,), (sum(NY) - len(NY) + 1,), MZ, reconstruction=reconstruction,
                              inviscid_scheme=inviscid_scheme)
    om, os_ = OracleRun(mb), OracleRun(sb)
    om.initialize()
    os_.initialize()
    return mb, om, os_


def _offsets(n):
    return np.cumsum([0] + [m - 1 for m in n])


@pytest.mark.parametrize("recon,scheme", [(2, 2), (2, 3), (3, 4), (1, 1)])
def test_split_grid_rhs_equals_whole_grid(recon, scheme):
    mb, om, os_ = _split_vs_whole(recon, scheme)
    om.compute_rhs()
    os_.compute_rhs()
    whole = os_.blocks[0].arrays["dq"]
    ox, oy = _offsets(NX), _offsets(NY)
    q = 0
    for bj, my in enumerate(NY):
        for bi, mx in enumerate(NX):
            got = om.blocks[q].arrays["dq"]
            sub = whole[:, :, oy[bj]:oy[bj] + my, ox[bi]:ox[bi] + mx]
            scale = np.max(np.abs(whole), axis=(1, 2, 3))
            err = np.max(np.abs(got - sub), axis=(1, 2, 3)) / scale
            assert np.all(err <= 1e-14), (q, err)
            q += 1


def test_initialize_fills_ghosts_from_neighbours():
    """After initialize every block's ghosted arrays equal the unsplit field
    on the same index range: the interface ghosts hold the neighbour's
    interior and the shared planes agree (averaging equal values)."""
    mb, om, os_ = _split_vs_whole(4, 2)
    g = mb.blocks[0].ngg
    whole = os_.blocks[0].arrays
    ox, oy = _offsets(NX), _offsets(NY)
    q = 0
    for bj, my in enumerate(NY):
        for bi, mx in enumerate(NX):
            for name in ("bv", "cv"):
                got = om.blocks[q].arrays[name]
                sub = whole[name][:, :, oy[bj]:oy[bj] + my + 2 * g, ox[bi]:ox[bi] + mx + 2 * g]
                # ghost rows/columns beyond the physical faces of the whole grid
                # differ only where the block face is physical in both
                assert np.array_equal(got, sub), (q, name)
            q += 1


def test_interface_exchange_after_steps_is_consistent():
    """After RK3 steps the shared planes carry one value in both blocks and
    the interface ghosts mirror the neighbour's interior. Lines shared by
    four blocks are left out: the exchange averages them pair by pair in
    face order, so the four copies differ (as in the reference)."""
    mb = ostc.case_multiblock(NX, NY, MZ, reconstruction=2, inviscid_scheme=2)
    o = OracleRun(mb)
    o.initialize()
    o.rk3_steps(3)
    g = mb.blocks[0].ngg
    ids = {(bi, bj): bj * len(NX) + bi for bj in range(len(NY)) for bi in range(len(NX))}
    for (bi, bj), q in ids.items():
        mx, my = NX[bi], NY[bj]
        # tangential ranges without the lines on the other direction's interfaces
        jr = slice(g + (1 if bj > 0 else 0), g + my - (1 if bj + 1 < len(NY) else 0))
        ir = slice(g + (1 if bi > 0 else 0), g + mx - (1 if bi + 1 < len(NX) else 0))
        kr = slice(g, -g)
        if bi + 1 < len(NX):
            a = o.blocks[q].arrays["bv"]
            b = o.blocks[ids[(bi + 1, bj)]].arrays["bv"]
            # shared plane i = mx-1 (left) == i = 0 (right)
            assert np.array_equal(a[:, kr, jr, g + mx - 1], b[:, kr, jr, g])
            for s in range(1, g + 1):
                assert np.array_equal(a[:, kr, jr, g + mx - 1 + s], b[:, kr, jr, g + s])
                assert np.array_equal(b[:, kr, jr, g - s], a[:, kr, jr, g + mx - 1 - s])
        if bj + 1 < len(NY):
            a = o.blocks[q].arrays["bv"]
            b = o.blocks[ids[(bi, bj + 1)]].arrays["bv"]
            assert np.array_equal(a[:, kr, g + my - 1, ir], b[:, kr, g, ir])
            for s in range(1, g + 1):
                assert np.array_equal(a[:, kr, g + my - 1 + s, ir], b[:, kr, g + s, ir])
                assert np.array_equal(b[:, kr, g - s, ir], a[:, kr, g + my - 1 - s, ir])
