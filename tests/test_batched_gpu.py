"""Tile-table launches (ostc_set_batching): every block of a context in one
persistent launch per kernel. Each cell sees the same operations in the same
order as with one launch per block, so the results must be bitwise equal:
RHS, residual histories and states after several RK3 steps, for the air
multi-block grid under each inviscid scheme and for the 9-species mixture,
with fused and split flux kernels and after tile-shape changes (which rebuild
the tables)."""
import numpy as np
import pytest

import ostc

pytestmark = pytest.mark.gpu

NX, NY, MZ = (17, 15, 12), (14, 17), 10
SCHEMES = {"aweno": (4, 2), "roe_muscl": (2, 2), "ausm_muscl": (2, 3), "hllc_nnd2": (3, 4)}


def _multiblock(name):
    recon, inv = SCHEMES[name]
    return ostc.case_multiblock(NX, NY, MZ, reconstruction=recon, inviscid_scheme=inv)


def _run(case, batched, steps=0, tiles=None):
    s, blocks = case.solver()
    if tiles:
        s.set_tiles(tiles)
    s.set_batching(batched)
    assert s.batching() == batched
    s.initialize()
    s.compute_rhs()
    out = {"dq": [b.download("dq") for b in blocks]}
    if steps:
        res, dts = s.rk3_steps(steps, history=True)
        out["res"], out["dt"] = res, dts
        for arr in ("bv", "cv"):
            out[arr] = [b.download(arr) for b in blocks]
    s.close()
    return out


def _equal(a, b):
    for k in a:
        if isinstance(a[k], list):
            for x, y in zip(a[k], b[k]):
                assert np.array_equal(x, y), k
        else:
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name", list(SCHEMES))
def test_batched_rhs_equals_per_block(name):
    case = _multiblock(name)
    _equal(_run(case, True), _run(case, False))


@pytest.mark.parametrize("name", ["aweno", "ausm_muscl"])
def test_batched_history_equals_per_block(name):
    case = _multiblock(name)
    _equal(_run(case, True, steps=6), _run(case, False, steps=6))


def test_batched_tile_shapes_and_split():
    case = _multiblock("hllc_nnd2")
    tiles = [(2 | 2 << 8, 2), (4 | 4 << 8, 3), (8 | 3 << 8, 1), (4 | 2 << 8, 2), (0, 0), (8, 2)]
    _equal(_run(case, True, steps=3, tiles=tiles), _run(case, False, steps=3, tiles=tiles))


def test_batched_mixture():
    case = ostc.case_mixing_layer(24, 20, 8)
    tiles = [(8 | 2 << 8, 1), (8 | 2 << 8, 2), (4 | 4 << 8, 3), (0, 0), (4 | 2 << 8, 2), (0, 0)]
    _equal(_run(case, True, steps=3), _run(case, False, steps=3))
    _equal(_run(case, True, steps=2, tiles=tiles), _run(case, False, steps=2, tiles=tiles))


def test_batching_toggle_on_one_context():
    case = _multiblock("ausm_muscl")
    s, blocks = case.solver()
    s.initialize()
    s.compute_rhs()
    ref = [b.download("dq") for b in blocks]
    for on in (True, False, True):
        s.set_batching(on)
        s.compute_rhs()
        for b, r in zip(blocks, ref):
            assert np.array_equal(b.download("dq"), r)
    s.close()


# boundary faces in batched launches: every face of every block (priority
# levels, then the periodic wraps) in one cooperative launch, in waves of faces
# with disjoint footprints; the per-face order of the reference stays wherever
# two faces of a block touch the same cells
BC_CASES = {
    "wall_farfield": lambda: ostc.case_bc_box("wall_farfield", 34, 27, 9),
    "subsonic": lambda: ostc.case_bc_box("subsonic", 34, 27, 9),
    "planar_wall_farfield": lambda: ostc.case_bc_box("wall_farfield", 34, 27, 1),
    "mixing_layer": lambda: ostc.case_mixing_layer(33, 26, 9, dx=1e-3, full_host=True),
    "uneven_sst": lambda: ostc.case_uneven_blocks(
        layout=ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False),
        rans_model=2),
}


@pytest.mark.parametrize("name", list(BC_CASES))
def test_batched_boundary_faces_equal_per_face(name):
    case = BC_CASES[name]
    _equal(_run(case(), True, steps=4), _run(case(), False, steps=4))


def test_boundary_waves_batch_the_faces_that_do_not_meet():
    """the wall-farfield box: its two far-field faces share an edge and both
    set their boundary layer (two waves), its two symmetry faces do not meet
    (one wave), so a batched stage has fewer launches than a per-face one"""
    case = ostc.case_bc_box("wall_farfield", 34, 27, 9)
    s, _ = case.solver()
    s.set_batching(True)
    s.initialize()
    n_batched = s.step_kernel_count(False)
    s.set_batching(False)
    n_face = s.step_kernel_count(False)
    s.close()
    assert n_batched < n_face, (n_batched, n_face)


def _stage_count(case, batched):
    s, _ = case.solver()
    s.set_batching(batched)
    n = s.step_kernel_count(False)
    s.close()
    return n


def test_faces_and_interfaces_are_one_launch_per_call():
    """batched, a step's launches do not depend on how many faces and
    interfaces the blocks have: a layout of 9 blocks and one of 37 blocks of
    the same flow give the same count (default tiles, one flux launch per
    sweep), and fewer than the per-face launches"""
    few = ostc.case_uneven_blocks(
        layout=ostc.block_layout(5, n_layers=2, n_cols=2, rows=(2, 2), extra_row=(0, 0), dims=(40, 30, 24),
                                 ranges=((8, 24), (8, 16), (8, 14)), anchors=False),
        rans_model=2)
    many = ostc.case_uneven_blocks(
        layout=ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False),
        rans_model=2)
    assert len(few.blocks) < len(many.blocks) and len(few.interfaces) < len(many.interfaces)
    n_few, n_many = _stage_count(few, True), _stage_count(many, True)
    assert n_few == n_many, (n_few, n_many)
    assert n_few < _stage_count(few, False)


def test_one_block_with_small_faces_batches_them_by_default():
    """one block: tile tables off by default; its faces (outflow and periodic,
    a few thousand points) in one wave launch, which launch-bound small faces
    favour. The step count is taken first, before any other call on the
    context (its graph capture must not hold the parameter upload), and the
    steps that follow equal those of per-face launches bit for bit"""
    case = lambda: ostc.case_mixing_layer(33, 26, 9, dx=1e-3, full_host=True)
    s, blocks = case().solver()
    assert not s.batching()
    n_default = s.step_kernel_count(False)
    s.initialize()
    res, dts = s.rk3_steps(4, history=True)
    got = {"res": res, "dt": dts, "bv": [b.download("bv") for b in blocks]}
    s.close()
    ref = _run(case(), False, steps=4)
    for k in ("res", "dt", "bv"):
        if isinstance(got[k], list):
            for x, y in zip(got[k], ref[k]):
                assert np.array_equal(x, y), k
        else:
            assert np.array_equal(got[k], ref[k]), k
    assert n_default < _stage_count(case(), False)
