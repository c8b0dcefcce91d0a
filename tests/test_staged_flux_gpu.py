"""The staged flux kernels (csrc/flux.cuh: flux_dir_staged, the sweep plane's
cells copied into a shared-memory tile before the faces are computed)
against the plane kernels, which the oracle and the reference build pin:
the same RHS bit for bit and the same steps, for every face they are built
for (primitive-variable reconstruction of first order, MUSCL and NND2 with
AUSM+, HLLC and Roe; the mixture; k-omega SST; several blocks walked by the
tile table; 2-D blocks), with tile shapes whose last tiles are partial at the
block edges. Blocks whose ghosted rows have an even length move their tiles
as 16-byte bulk copies, the others as 8-byte cp.async: both are covered (the
"_even" cases and their odd twins). The split inviscid and viscous kernels
are staged alike.
"""
import numpy as np
import pytest

import ostc
from planar_cases import planar_sst

pytestmark = pytest.mark.gpu

PLANE = [(4 | 2 << 8, 2), (8 | 2 << 8, 2), (4 | 2 << 8, 3)]


def staged(chunks=(2, 3, 2)):
    return [(8 | 2 << 8 | 1 << 16, chunks[d]) for d in range(3)]


def _mixing(mx=37, **kw):
    return ostc.case_mixing_layer(mx, 29, 19, dx=1e-3, full_host=True, **kw)


def _scheme(case, reconstruction=None, inviscid_scheme=None):
    if reconstruction is not None:
        case.scheme.reconstruction = reconstruction
    if inviscid_scheme is not None:
        case.scheme.inviscid_scheme = inviscid_scheme
    return case


CASES = {
    "mixing_muscl_ausm": lambda: _mixing(),
    "mixing_muscl_hllc": lambda: _scheme(_mixing(), inviscid_scheme=4),
    "mixing_nnd2_ausm": lambda: _scheme(_mixing(), reconstruction=3),
    "mixing_first_order": lambda: _scheme(_mixing(), reconstruction=1),
    "mixing_muscl_roe": lambda: _scheme(_mixing(), inviscid_scheme=2),
    "mixing_sst_wall": lambda: _mixing(rans_model=2, wall=True),
    "vortex_muscl_hllc": lambda: ostc.case_vortex(45, 38, 11, reconstruction=2, inviscid_scheme=4),
    "uneven_sst_blocks": lambda: ostc.case_uneven_blocks(
        layout=ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False),
        rans_model=2),
    "planar_sst": lambda: planar_sst(),
    "planar_mixing": lambda: ostc.case_mixing_layer(41, 23, 1, full_host=True),
    "mixing_muscl_ausm_even": lambda: _mixing(38),
    "mixing_muscl_roe_even": lambda: _scheme(_mixing(38), inviscid_scheme=2),
    "mixing_sst_wall_even": lambda: _mixing(38, rans_model=2, wall=True),
    "vortex_muscl_hllc_even": lambda: ostc.case_vortex(46, 38, 11, reconstruction=2, inviscid_scheme=4),
    "planar_mixing_even": lambda: ostc.case_mixing_layer(42, 23, 1, full_host=True),
    "even_blocks": lambda: ostc.case_uneven_blocks(
        layout=[((0, 0, 0), (20, 14, 10)), ((19, 0, 0), (40, 14, 10))], rans_model=2),
}


def test_even_rows_take_the_bulk_copies():
    """the zone flag that selects bulk copies: even ghosted rows and aligned planes"""
    for name, even in (("mixing_muscl_ausm", False), ("mixing_muscl_ausm_even", True)):
        b = CASES[name]().blocks[0]
        assert ((b.mx + 2 * b.ngg) % 2 == 0) == even


def _run(case, tiles, split=False, steps=0):
    s, blocks = case.solver()
    s.set_tiles(tiles)
    if split:  # the separate inviscid and viscous kernels, both staged like the fused one
        for d in range(3):
            s.set_tile(d + 3, *tiles[d])
    s.initialize()
    s.compute_rhs()
    dq = [b.download("dq") for b in blocks]
    hist = None
    if steps:
        s.initialize()
        hist = s.rk3_steps(steps, history=True)
        hist = (hist, [b.download("bv") for b in blocks])
    s.close()
    return dq, hist


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("chunks", [(2, 3, 2), (1, 1, 5)])
def test_staged_rhs_is_the_plane_rhs(name, chunks):
    ref, _ = _run(CASES[name](), PLANE)
    got, _ = _run(CASES[name](), staged(chunks))
    for a, b in zip(got, ref):
        assert np.array_equal(a, b), float(np.nanmax(np.abs(a - b)))


def test_staged_split_kernels():
    case = CASES["mixing_muscl_hllc"]
    ref, _ = _run(case(), PLANE)
    got, _ = _run(case(), staged(chunks=(1, 5, 3)), split=True)
    # the split kernels add the inviscid and viscous differences separately:
    # the same terms in another order, so equal to rounding
    for a, b in zip(got, ref):
        scale = np.max(np.abs(b), axis=tuple(range(1, b.ndim)), keepdims=True)
        assert np.max(np.abs(a - b) / np.where(scale > 0, scale, 1)) < 1e-12


@pytest.mark.parametrize("name", ["mixing_muscl_ausm", "mixing_muscl_ausm_even"])
def test_staged_steps_are_the_plane_steps(name):
    case = CASES[name]
    _, (h_ref, bv_ref) = _run(case(), PLANE, steps=4)
    _, (h_got, bv_got) = _run(case(), staged(), steps=4)
    assert np.array_equal(h_got[0], h_ref[0]) and np.array_equal(h_got[1], h_ref[1])
    for a, b in zip(bv_got, bv_ref):
        assert np.array_equal(a, b)


def test_staged_tiles_need_eight_rows():
    case = CASES["mixing_muscl_ausm"]()
    s, _ = case.solver()
    with pytest.raises(ostc.OstcError):
        s.set_tile(0, 4 | 2 << 8 | 1 << 16, 2)
    s.close()


def test_staged_tiles_refused_for_aweno():
    case = ostc.case_vortex(24, 20, 8)
    s, _ = case.solver()
    s.set_tiles(staged())
    s.initialize()
    with pytest.raises(ostc.OstcError):
        s.compute_rhs()
    s.close()
