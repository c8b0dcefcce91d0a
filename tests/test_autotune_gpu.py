"""The flux autotuner behind the C ABI (ostc_autotune, api.cu): it leaves a
runnable tile on every direction, reports a positive time per launch, keeps
the flow state untouched, and the right-hand side with its tiles equals the
one with the default tiles (bit for bit when it keeps the fused kernels, to
rounding when a direction's flux runs as separate inviscid and viscous
kernels); AWENO never gets a staged tile."""
import numpy as np
import pytest

import ostc

pytestmark = pytest.mark.gpu


def _rhs(case, tune):
    s, blocks = case.solver()
    s.initialize()
    bv0 = blocks[0].download("bv")
    best = s.autotune(warmup=1, reps=2) if tune else None
    assert np.array_equal(blocks[0].download("bv"), bv0)
    s.initialize()
    s.compute_rhs()
    out = [b.download("dq") for b in blocks]
    tiles = s.tiles()
    s.close()
    return out, best, tiles


@pytest.mark.parametrize("name", ["mixing", "vortex_aweno", "sst_blocks"])
def test_autotuned_tiles_give_the_same_rhs(name):
    make = {
        "mixing": lambda: ostc.case_mixing_layer(38, 29, 19, dx=1e-3, full_host=True),
        "vortex_aweno": lambda: ostc.case_vortex(40, 32, 10),
        "sst_blocks": lambda: ostc.case_uneven_blocks(
            layout=ostc.block_layout(5, dims=(40, 30, 32), ranges=((8, 20), (8, 14), (8, 10)), anchors=False),
            rans_model=2),
    }[name]
    ref, _, _ = _rhs(make(), False)
    got, best, tiles = _rhs(make(), True)
    assert all(best[d][0] > 0 for d in range(3)), best
    if name == "vortex_aweno":
        assert all((r >> 16) == 0 for r, _ in tiles[:3]), tiles
    split = any(r != 0 for r, _ in tiles[3:])
    for a, b in zip(got, ref):
        if split:
            scale = np.max(np.abs(b), axis=tuple(range(1, b.ndim)), keepdims=True)
            assert np.max(np.abs(a - b) / np.where(scale > 0, scale, 1)) < 1e-12
        else:
            assert np.array_equal(a, b)
