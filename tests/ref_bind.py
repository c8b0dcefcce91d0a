"""ctypes binding of the reference's own CUDA kernels driven by
oracle/ref_cuda_harness.cu (oracle/_ref/libostc_ref_cuda.so, built from the
reference sources by oracle/build_ref.sh). Test and measurement
infrastructure: the tight GPU oracle and the reference-build timing."""
import ctypes as C
from pathlib import Path

import numpy as np

import ostc

REPO = Path(__file__).resolve().parents[1]
REF_CUDA = REPO / "oracle" / "_ref" / "libostc_ref_cuda.so"
_r = None


def available():
    return REF_CUDA.exists()


def ref():
    global _r
    if _r is None:
        L = C.CDLL(str(REF_CUDA))
        vp = C.c_void_p
        d = C.POINTER(C.c_double)
        L.ref_create.argtypes = [C.POINTER(ostc.Config), C.POINTER(ostc.Param), C.POINTER(ostc.Zone),
                                 C.POINTER(ostc.BcFaceC), C.c_int, C.POINTER(vp)]
        L.ref_create.restype = C.c_int
        L.ref_create_multi.argtypes = [C.POINTER(ostc.Config), C.POINTER(ostc.Param), C.POINTER(ostc.Zone), C.c_int,
                                       C.POINTER(ostc.BcFaceC), C.c_int, C.POINTER(ostc.IfaceC), C.c_int,
                                       C.POINTER(vp)]
        L.ref_create_multi.restype = C.c_int
        L.ref_download_block.argtypes = [vp, C.c_int, C.c_char_p, d]
        L.ref_download_block.restype = C.c_int
        for n in ("ref_initialize", "ref_rhs"):
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = C.c_int
        L.ref_steps.argtypes = [vp, C.c_int, d, d]
        L.ref_steps.restype = C.c_int
        L.ref_steady_steps.argtypes = [vp, C.c_int, d]
        L.ref_steady_steps.restype = C.c_int
        L.ref_time_steps.argtypes = [vp, C.c_int]
        L.ref_time_steps.restype = C.c_double
        L.ref_download.argtypes = [vp, C.c_char_p, d]
        L.ref_download.restype = C.c_int
        L.ref_zone_view.argtypes = [vp, C.c_int, C.POINTER(ostc.Zone)]
        L.ref_zone_view.restype = C.c_int
        L.ref_metric.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, d, d, d, d, vp]
        L.ref_metric.restype = C.c_int
        ip = C.POINTER(C.c_int)
        L.ref_mesh_read.argtypes = [C.c_char_p, C.c_int, C.c_double, C.POINTER(vp)]
        L.ref_mesh_read.restype = C.c_int
        L.ref_mesh_counts.argtypes = [vp, ip, ip]
        L.ref_mesh_counts.restype = C.c_int
        L.ref_mesh_block.argtypes = [vp, C.c_int, ip, d, d, d, d, vp]
        L.ref_mesh_block.restype = C.c_int
        L.ref_mesh_boundaries.argtypes = [vp, C.c_int, ip, ip]
        L.ref_mesh_boundaries.restype = C.c_int
        L.ref_mesh_inner.argtypes = [vp, C.c_int, ip, ip]
        L.ref_mesh_inner.restype = C.c_int
        _r = L
    return _r


class RefCudaRun:
    """The reference build on all blocks of a Case (single-rank); blocks
    exchange through the reference's inner_communication kernel."""

    def __init__(self, case):
        self.case = case
        self.blocks = case.blocks
        self.block = case.blocks[0]
        self.param, self._keep = ostc.make_param(case.scheme, case.mech)
        self.config = ostc.make_config(case.scheme)
        self.zones = (ostc.Zone * len(case.blocks))(*[b.zone() for b in case.blocks])
        self.faces = (ostc.BcFaceC * max(len(case.faces), 1))(*case.faces)
        ifs = list(getattr(case, "interfaces", []) or [])
        self.ifaces = (ostc.IfaceC * max(len(ifs), 1))(*ifs)
        h = C.c_void_p()
        st = ref().ref_create_multi(C.byref(self.config), C.byref(self.param), self.zones, len(case.blocks),
                                    self.faces, len(case.faces), self.ifaces, len(ifs), C.byref(h))
        if st != 0:
            raise RuntimeError("ref_create_multi -> %d" % st)
        self.h = h

    def initialize(self):
        assert ref().ref_initialize(self.h) == 0

    def compute_rhs(self):
        assert ref().ref_rhs(self.h) == 0

    def rk3_steps(self, n):
        res = (C.c_double * (4 * n))()
        dts = (C.c_double * n)()
        assert ref().ref_steps(self.h, n, res, dts) == 0
        return np.array(res).reshape(n, 4), np.array(dts)

    def steady_steps(self, n):
        res = (C.c_double * (4 * n))()
        assert ref().ref_steady_steps(self.h, n, res) == 0
        return np.array(res).reshape(n, 4)

    def time_steps(self, n):
        return ref().ref_time_steps(self.h, n)

    def zone_view(self, block=0):
        """block's device arrays in the reference build as an ostc_zone
        (include/ostc_reference_shim.h): this library can run on them"""
        z = ostc.Zone()
        assert ref().ref_zone_view(self.h, block, C.byref(z)) == 0
        return z

    def download(self, name, block=0):
        b = self.blocks[block]
        P = ostc.plane_shape(b.mx, b.my, b.mz, b.ngg)
        I = ostc.plane_shape(b.mx, b.my, b.mz, 0)
        Q = ostc.plane_shape(b.mx, b.my, b.mz, getattr(b, "dq_ngg", 0))
        shapes = {"bv": (6,) + P, "sv": (b.n_spec + b.n_turb,) + P, "cv": (b.n_var,) + P, "dq": (b.n_var,) + Q,
                  "mul": P, "thermal_conductivity": P, "vel": P, "acoustic_speed": P, "rho_D": (b.n_spec,) + P,
                  "mut": P, "turb_therm_cond": P}
        out = np.zeros(shapes[name])
        assert ref().ref_download_block(self.h, block, name.encode(), out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out


def metric(mx, my, mz, ngg, x, y, z):
    """the reference's Block::compute_jac_metric on coordinates with ngg+1
    ghost layers: (jac, metric) as ghosted arrays (metric in ostc.METRIC_DTYPE)"""
    shape = ostc.plane_shape(mx, my, mz, ngg)
    jac = np.zeros(shape)
    met = np.zeros(shape, dtype=ostc.METRIC_DTYPE)
    d = C.POINTER(C.c_double)
    xs, ys, zs = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    st = ref().ref_metric(mx, my, mz, ngg, xs.ctypes.data_as(d), ys.ctypes.data_as(d), zs.ctypes.data_as(d),
                          jac.ctypes.data_as(d), met.ctypes.data)
    if st != 0:
        raise RuntimeError("ref_metric -> %d" % st)
    return jac, met


def mesh(directory, ngg, grid_scale):
    """the reference's own cfd::Mesh (src/Mesh.cpp:550-588) from the files
    under directory/input_files: per block a dict of extents, x, y, z, jac,
    metric (ngg ghost layers), the registered boundary faces (rows of
    range_start, range_end, face, direction, label) and inner faces (rows of
    range_start, range_end, target_start, loop_dir, target_loop_dir, src_tar,
    n_point, face, direction, target_block, target_face); and the dimension"""
    h = C.c_void_p()
    st = ref().ref_mesh_read(str(directory).encode(), ngg, grid_scale, C.byref(h))
    if st != 0:
        raise RuntimeError("ref_mesh_read -> %d" % st)
    nb, dim = C.c_int(), C.c_int()
    ref().ref_mesh_counts(h, C.byref(nb), C.byref(dim))
    out = []
    d = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    for b in range(nb.value):
        dims = (C.c_int * 3)()
        ref().ref_mesh_block(h, b, dims, None, None, None, None, None)
        mx, my, mz = list(dims)
        shape = ostc.plane_shape(mx, my, mz, ngg)
        x, y, z, jac = (np.zeros(shape) for _ in range(4))
        met = np.zeros(shape, dtype=ostc.METRIC_DTYPE)
        ref().ref_mesh_block(h, b, dims, x.ctypes.data_as(d), y.ctypes.data_as(d), z.ctypes.data_as(d),
                             jac.ctypes.data_as(d), met.ctypes.data)
        n = C.c_int()
        ref().ref_mesh_boundaries(h, b, C.byref(n), None)
        bnd = np.zeros((n.value, 9), dtype=np.int32)
        ref().ref_mesh_boundaries(h, b, C.byref(n), bnd.ctypes.data_as(ip))
        ref().ref_mesh_inner(h, b, C.byref(n), None)
        inner = np.zeros((n.value, 25), dtype=np.int32)
        ref().ref_mesh_inner(h, b, C.byref(n), inner.ctypes.data_as(ip))
        out.append({"dims": (mx, my, mz), "x": x, "y": y, "z": z, "jac": jac, "metric": met, "boundaries": bnd,
                    "inner": inner})
    return out, dim.value
