"""A run on a mesh read from the reference's input-file formats: the 2-D
two-block step (mesh_files.step_2d, the layout of the reference's shipped
grid) with its conditions from a setup file in the reference's syntax (a
Mach 2 air inflow, a second inflow on the lower part of the wider block's
i-min face, isothermal walls, an outflow), through ostc_mesh_read,
ostc.boundary_setup and the interface exchange: 5 RK3 steps against the CPU
oracle and the reference's own kernels on the same blocks, faces and
interfaces."""
import numpy as np
import pytest

import mesh_files
import ostc
import ref_bind
from oracle_bind import OracleRun, normwise

pytestmark = pytest.mark.gpu

SETUP = """array   string  boundary_conditions {
    freestream jet wall
}
struct  freestream {
    string  type            =   inflow
    int     label           =   5
    real    temperature     =   300
    real    mach            =   2
    real    pressure        =   101325
    real    u               =   1
    real    v               =   0
    real    w               =   0
}
struct  jet {
    string  type            =   inflow
    int     label           =   9
    real    temperature     =   250
    real    mach            =   1.2
    real    pressure        =   101325
    real    u               =   1
    real    v               =   0
    real    w               =   0
}
struct  wall {
    string  type            =   wall
    int     label           =   2
    string  thermal_type    =   isothermal
    real    temperature     =   300
}
"""


def _case(tmp_path):
    paths = mesh_files.step_2d(tmp_path)
    scheme = ostc.Scheme(mix_model=ostc.MIX_AIR, inviscid_scheme=3, reconstruction=2, viscous_order=2, cfl=0.4)
    ng = scheme.ngg
    mesh = ostc.read_mesh(*paths, ngg=ng, grid_scale=0.001)
    (tmp_path / "setup.txt").write_text(SETUP)
    setup = ostc.read_setup(tmp_path / "setup.txt")
    faces = ostc.boundary_setup(setup, mesh.faces, ng)
    inf = ostc.inflow_state(setup["freestream"])
    blocks = []
    for (mx, my, mz), jac, met in zip(mesh.dims, mesh.jac, mesh.metric):
        b = ostc.HostBlock.allocate(mx, my, mz, ng, 5, 0)
        b.arrays["jac"][...] = jac
        b.arrays["metric"][...] = met
        bv = b.arrays["bv"]
        bv[0], bv[1], bv[2], bv[3] = inf["density"], inf["u"], 0.0, 0.0
        bv[4], bv[5] = inf["pressure"], inf["temperature"]
        blocks.append(b)
    c = ostc.Case("step_2d", scheme, None, blocks, faces, 5)
    c.interfaces = mesh.interfaces
    return c


def test_step_mesh_against_oracle_and_reference_build(tmp_path):
    case = _case(tmp_path)
    assert [f.type_label for f in case.faces] == [ostc.BC_WALL, ostc.BC_WALL, ostc.BC_INFLOW, ostc.BC_WALL,
                                                 ostc.BC_OUTFLOW, ostc.BC_WALL, ostc.BC_INFLOW]
    n = 5
    o = OracleRun(case)
    o.initialize()
    res_o, dt_o = o.rk3_steps(n)
    s, blocks = case.solver()
    s.initialize()
    res_g, dt_g = s.rk3_steps(n, history=True)
    assert np.max(np.abs(dt_g - dt_o) / dt_o) <= 1e-9
    assert np.max(np.abs(res_g - res_o) / res_o) <= 1e-9
    for b in range(len(blocks)):
        assert max(normwise(blocks[b].download("bv"), o.blocks[b].arrays["bv"])) <= 1e-9, b
    if ref_bind.available():
        r = ref_bind.RefCudaRun(case)
        r.initialize()
        res_r, dt_r = r.rk3_steps(n)
        assert np.max(np.abs(dt_g - dt_r) / dt_r) <= 1e-9
        for b in range(len(blocks)):
            assert max(normwise(blocks[b].download("bv"), r.download("bv", b))) <= 1e-9, b
    s.close()
