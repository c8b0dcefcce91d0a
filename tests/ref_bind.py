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
        L.ref_metric.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, d, d, d, d, vp]
        L.ref_metric.restype = C.c_int
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
