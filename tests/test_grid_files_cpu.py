"""The grid pre-processing (ostc_mesh_read: grid, boundary and inner-face
files, face registration, ghost grid, metrics) against the reference's own
cfd::Mesh run on the same files (src/Mesh.cpp:550-588, compiled from the
reference sources into oracle/_ref): coordinates with their ghost layers,
Jacobians and metric records bit for bit, and the registered boundary and
inner faces field by field. On the CPU (both are host code); skipped where
the reference build is absent. The reference's shipped 2-block grid is
checked too where its input files are present. The setup-file reader is
checked on its own."""
import os
from pathlib import Path

import numpy as np
import pytest

import mesh_files
import ostc
import ref_bind

needs_ref = pytest.mark.skipif(not ref_bind.available(), reason="reference build (oracle/_ref) not present")


def _compare(directory, paths, ngg, scale):
    ours = ostc.read_mesh(*paths, ngg=ngg, grid_scale=scale)
    ref, dim = ref_bind.mesh(directory, ngg, scale)
    assert ours.dimension == dim and len(ours.dims) == len(ref)
    fq = iq = 0
    for b, rb in enumerate(ref):
        assert ours.dims[b] == rb["dims"]
        for a, name in enumerate("xyz"):
            assert np.array_equal(ours.coords[b][a], rb[name]), (b, name)
        assert np.array_equal(ours.jac[b], rb["jac"])
        assert np.array_equal(ours.metric[b]["m"], rb["metric"]["m"])
        for row in rb["boundaries"]:
            f = ours.faces[fq]
            fq += 1
            assert f.block == b
            assert list(f.range_start) + list(f.range_end) + [f.face, f.direction, f.type_label] == list(row)
        for row in rb["inner"]:
            f = ours.interfaces[iq]
            iq += 1
            got = (list(f.range_start) + list(f.range_end) + list(f.target_start) + list(f.loop_dir) +
                   list(f.target_loop_dir) + list(f.src_tar) + list(f.n_point) + [f.face, f.direction, f.target])
            assert f.block == b and got == list(row[:24]), (b, got, list(row))
    assert fq == len(ours.faces) and iq == len(ours.interfaces)
    return ours


@needs_ref
@pytest.mark.parametrize("ngg", [2, 3])
def test_two_block_step_2d(tmp_path, ngg):
    paths = mesh_files.step_2d(tmp_path)
    m = _compare(tmp_path, paths, ngg, 0.001)
    assert len(m.faces) == 7 and len(m.interfaces) == 2


@needs_ref
@pytest.mark.parametrize("ngg", [2, 3])
def test_stacked_blocks_3d(tmp_path, ngg):
    paths = mesh_files.stacked_3d(tmp_path)
    m = _compare(tmp_path, paths, ngg, 1.0)
    assert m.dimension == 3 and len(m.interfaces) == 2


REF_INPUT = Path(os.environ.get("OSTC_REFERENCE_DIR", "/root/reference")) / "input_files"


@needs_ref
@pytest.mark.skipif(not (REF_INPUT / "grid" / "grid   0.grd").exists(), reason="the reference's input files are absent")
def test_shipped_two_block_grid():
    """the reference's own input_files (2-D, 201x100 and 201x163 nodes)"""
    bc = REF_INPUT / "boundary_condition"
    paths = (REF_INPUT / "grid" / "grid   0.grd", bc / "boundary   0.txt", bc / "inner   0.txt")
    m = _compare(REF_INPUT.parent, paths, 2, 0.001)
    assert m.dims == [(201, 100, 1), (201, 163, 1)]


def test_malformed_files_are_refused(tmp_path):
    g, b, i = mesh_files.step_2d(tmp_path)
    b.write_text(b.read_text().splitlines()[0] + "\n")  # a face count with no faces
    with pytest.raises(ostc.OstcError) as e:
        ostc.read_mesh(g, b, i)
    assert e.value.status == ostc.ERR_IO
    with pytest.raises(ostc.OstcError):
        ostc.read_mesh(tmp_path / "missing.grd", b)


def test_setup_file_reader(tmp_path):
    """Parameter::read_one_file's syntax (src/Parameter.cpp:53-163)"""
    p = tmp_path / "5_boundary_condition.txt"
    p.write_text("""// comment
array   string  boundary_conditions {
    freestream wall
}
int     n = 3   // trailing comment
real    gridScale = 0.001
bool    parallel = 0
struct  freestream {
    string  type            =   inflow
    int     label           =   5
    real    temperature     =   300
    real    mach            =   2
    real    pressure        =   101325
}
struct  wall {
    string  type            =   wall
    int     label           =   2
    string  thermal_type    =   isothermal
    real    temperature     =   294.4
}
""")
    s = ostc.read_setup(p)
    assert s["boundary_conditions"] == ["freestream", "wall"] and s["n"] == 3 and s["gridScale"] == 0.001
    assert s["parallel"] is False and s["freestream"]["mach"] == 2.0 and s["wall"]["thermal_type"] == "isothermal"
    st = ostc.inflow_state(s["freestream"])
    ref = ostc.air_state(2.0, 300.0, 101325.0)
    assert abs(st["velocity"] - ref["u"]) <= 1e-12 * ref["u"] and abs(st["density"] - ref["density"]) <= 1e-15
