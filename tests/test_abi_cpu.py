"""The C ABI surface without a GPU: the library loads, exports every
function that include/ostc.h declares, and rejects bad arguments before
touching the device."""
import ctypes as C
import re
from pathlib import Path

import ostc

REPO = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"\b(ostc_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_symbols_exported():
    lib = ostc.lib()
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in ostc.lib().ostc_version()


def test_create_rejects_null():
    ctx = C.c_void_p()
    assert ostc.lib().ostc_create(None, None, None, 0, None, 0, C.byref(ctx)) == ostc.ERR_INVALID_ARG


def test_create_rejects_bad_face():
    case = ostc.case_vortex(16, 12, 8)
    p, keep = ostc.make_param(case.scheme, None)
    cfg = ostc.make_config(case.scheme)
    zones = (ostc.Zone * 1)(case.blocks[0].zone())  # host pointers: validation runs before any device use
    bad = ostc.bc_face(0, ostc.BC_INFLOW, 0, -1, (16, 12, 8), 3)
    bad.range_start[0] = 3
    faces = (ostc.BcFaceC * 1)(bad)
    ctx = C.c_void_p()
    assert ostc.lib().ostc_create(C.byref(cfg), C.byref(p), zones, 1, faces, 1, C.byref(ctx)) == ostc.ERR_INVALID_ARG


def test_create_rejects_unsupported_scheme():
    case = ostc.case_vortex(16, 12, 8)
    s = case.scheme
    p, keep = ostc.make_param(s, None)
    p.turbulence = 1  # RANS with a model other than SST (rans_model 0): refused before any device use
    cfg = ostc.make_config(s)
    zones = (ostc.Zone * 1)(case.blocks[0].zone())
    ctx = C.c_void_p()
    assert ostc.lib().ostc_create(C.byref(cfg), C.byref(p), zones, 1, None, 0, C.byref(ctx)) == ostc.ERR_UNSUPPORTED


def _create(case, p, cfg):
    zones = (ostc.Zone * len(case.blocks))(*[b.zone() for b in case.blocks])
    ctx = C.c_void_p()
    return ostc.lib().ostc_create(C.byref(cfg), C.byref(p), zones, len(case.blocks), None, 0, C.byref(ctx))


def test_create_rejects_sst_with_split_chemistry():
    """SST with the operator-split chemistry (chem_mode 1 / 2) is not built"""
    case = ostc.case_mixing_layer(12, 10, 6, full_host=True, rans_model=2)
    p, keep = ostc.make_param(case.scheme, case.mech)
    case.scheme.chem_mode = 1
    assert _create(case, p, ostc.make_config(case.scheme)) == ostc.ERR_UNSUPPORTED


def test_create_rejects_inconsistent_sst_counts():
    """k, omega must follow the species: n_var = 7 + n_spec, i_turb_cv = 5 + n_spec"""
    case = ostc.case_mixing_layer(12, 10, 6, full_host=True, rans_model=2)
    p, keep = ostc.make_param(case.scheme, case.mech)
    p.i_turb_cv = 5
    assert _create(case, p, ostc.make_config(case.scheme)) == ostc.ERR_INVALID_ARG


def test_create_rejects_mixed_2d_and_3d_blocks():
    """a problem is 2-D when its first block has mz == 1; every block must agree"""
    planar = ostc.case_vortex(16, 12, 1)
    solid = ostc.case_vortex(16, 12, 8)
    case = ostc.Case("mixed", planar.scheme, None, [planar.blocks[0], solid.blocks[0]], [], 1)
    p, keep = ostc.make_param(case.scheme, None)
    assert _create(case, p, ostc.make_config(case.scheme)) == ostc.ERR_INVALID_ARG


def test_metric_of_cartesian_grid():
    b = ostc.HostBlock.allocate(8, 7, 6, 2, 5, 0)
    x, y, z = ostc.grid_coordinates(8, 7, 6, 3, 1e-3, warp=0.0)
    ostc.fill_metric(b, x, y, z)
    m = b.arrays["metric"]["m"]
    assert abs(b.arrays["jac"].max() - 1e-9) < 1e-21 and abs(b.arrays["jac"].min() - 1e-9) < 1e-21
    assert abs(m[..., 0].max() - 1e3) < 1e-9 and abs(m[..., 1]).max() == 0
