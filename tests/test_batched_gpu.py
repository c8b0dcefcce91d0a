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
