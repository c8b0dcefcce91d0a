"""2-D (mz == 1) workloads and their uniform-in-k 3-D twins. Test
infrastructure.

A 2-D block of the reference runs on one k plane: its k ghost planes are
copies of k = 0 (eliminate_k_gradient, src/FieldOperation.cuh:372-400), the
z fluxes are skipped (src/InviscidScheme.cu:34, src/SchemeSelector.cuh:64)
and the grid's k spacing is one (src/Mesh.cpp:840-854). The same plane
repeated mz times with unit k spacing and periodic k faces is a 3-D block on
which every k difference is exactly zero, so both must evolve alike at a
fixed dt when the flux has no dimension-dependent term (every scheme but
Roe's entropy fix, src/Roe.cu:79-85). Single blocks only: with interfaces
the 3-D twin's periodic k ghosts are filled before the interface exchange
(BoundCond.cuh:673-822 then DataCommunication.cuh:27-56), a stage later
than the 2-D copy."""
import copy

import numpy as np

import ostc


def planar_sst(mx=25, my=21, dx=1e-4):
    """one 2-D block of the walled SST workload (case_uneven_blocks)"""
    return ostc.case_uneven_blocks(layout=[((0, 0, 0), (mx, my, 1))], dx=dx, rans_model=2)


def planar_cases():
    """name -> builder of the single-block 2-D workloads: 25 x 21 points, a
    size at which the reference's block reductions are defined (its min and
    sum leave a shared slot unwritten when the last block holds 32, 64 or 96
    points, MyAtomic.cuh:12-64)"""
    return {
        "vortex_muscl_hllc": lambda: ostc.case_vortex(25, 21, 1, reconstruction=2, inviscid_scheme=4),
        "vortex_muscl_ausm": lambda: ostc.case_vortex(25, 21, 1, reconstruction=2, inviscid_scheme=3),
        "vortex_aweno": lambda: ostc.case_vortex(25, 21, 1),
        "vortex_muscl_roe": lambda: ostc.case_vortex(25, 21, 1, reconstruction=2, inviscid_scheme=2),
        "wall_farfield": lambda: ostc.case_bc_box("wall_farfield", 25, 21, 1),
        "subsonic": lambda: ostc.case_bc_box("subsonic", 25, 21, 1),
        "mixing_h2air": lambda: ostc.case_mixing_layer(25, 21, 1, full_host=True),
        "sst_wall": lambda: planar_sst(),
        "sst_h2air_wall": lambda: ostc.case_mixing_layer(25, 21, 1, full_host=True, rans_model=2, wall=True),
    }


def _tile_k(a, ng, mz):
    """repeat the plane k = 0 (ghosted index ng) of a ghosted array over mz + 2 ng planes"""
    plane = a[..., ng:ng + 1, :, :]
    reps = [1] * a.ndim
    reps[-3] = mz + 2 * ng
    return np.tile(plane, reps)


def extrude(case, mz=4, dt=None):
    """The uniform-in-k 3-D twin of a single-block 2-D case: mz copies of its
    plane (state, Jacobian, metric, wall distance), the 2-D faces widened over
    k, periodic k faces; the same scheme with a fixed dt (dt or the case's)."""
    assert len(case.blocks) == 1 and case.blocks[0].mz == 1
    b = case.blocks[0]
    ng = b.ngg
    nb = ostc.HostBlock.allocate(b.mx, b.my, mz, ng, b.n_var, b.n_spec, full=True, dq_ngg=b.dq_ngg,
                                 n_turb=b.n_turb)
    for name in ("bv", "sv", "jac", "metric", "wall_distance"):
        if name in b.arrays and b.arrays[name].size:
            nb.arrays[name][...] = _tile_k(b.arrays[name], ng, mz)
    faces = []
    for f in case.faces:
        g = type(f).from_buffer_copy(f)
        wall = f.type_label == ostc.BC_WALL
        g.range_start[2], g.range_end[2] = (0, mz - 1) if wall else (-ng, mz - 1 + ng)
        faces.append(g)
    ext = (b.mx, b.my, mz)
    faces += [ostc.bc_face(0, ostc.BC_PERIODIC, 2, -1, ext, ng), ostc.bc_face(0, ostc.BC_PERIODIC, 2, 1, ext, ng)]
    s = copy.deepcopy(case.scheme)
    if dt is not None:
        s.fixed_time_step, s.dt = 1, dt
    return ostc.Case(case.name + "_extruded%d" % mz, s, case.mech, [nb], faces, case.steps)


def with_fixed_dt(case, dt):
    s = copy.deepcopy(case.scheme)
    s.fixed_time_step, s.dt = 1, dt
    c = ostc.Case(case.name, s, case.mech, case.blocks, case.faces, case.steps)
    c.interfaces = list(getattr(case, "interfaces", []) or [])
    return c


def k_plane(a, ng, k=0):
    """plane k of a ghosted array (variables first)"""
    return a[..., ng + k, :, :]
