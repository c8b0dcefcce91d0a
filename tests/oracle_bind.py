"""ctypes binding of the CPU oracle (oracle/liboracle.so). Test
infrastructure: used only by tests/, the smoke check and bench.py's CPU
baseline legs, always as the checker."""
import ctypes as C
from pathlib import Path

import numpy as np

import ostc

REPO = Path(__file__).resolve().parents[1]
ORACLE = REPO / "oracle" / "liboracle.so"
_o = None


def oracle():
    global _o
    if _o is None:
        if not ORACLE.exists():
            raise RuntimeError("oracle/liboracle.so missing: run __graft_entry__.build()")
        L = C.CDLL(str(ORACLE))
        P, Z, F, G = C.POINTER(ostc.Param), C.POINTER(ostc.Zone), C.POINTER(ostc.BcFaceC), C.POINTER(ostc.Config)
        d = C.POINTER(C.c_double)
        sig = {
            "oracle_compute_cv_from_bv": ([P, Z], C.c_int),
            "oracle_compute_rhs": ([P, Z], C.c_int),
            "oracle_flux_scale": ([P, Z, d], C.c_int),
            "oracle_global_time_step": ([P, Z, C.c_int], C.c_double),
            "oracle_update_cv_and_bv_rk": ([P, Z, C.c_double, C.c_int], C.c_int),
            "oracle_apply_boundary_conditions": ([P, Z, C.c_int, F, C.c_int, C.c_int], C.c_int),
            "oracle_update_physical_properties": ([P, Z], C.c_int),
            "oracle_initialize": ([G, P, Z, C.c_int, F, C.c_int], C.c_int),
            "oracle_rk3_steps": ([G, P, Z, C.c_int, F, C.c_int, C.c_int, d, d], C.c_int),
            "oracle_chemical_source": ([P, C.c_double, C.c_double, d, d], C.c_int),
            "oracle_enthalpy_cp": ([P, C.c_double, d, d], C.c_int),
            "oracle_transport": ([P, C.c_double, C.c_double, C.c_double, d, d, d, d], C.c_int),
            "oracle_set_threads": ([C.c_int], None),
            "oracle_set_interfaces": ([C.POINTER(ostc.IfaceC), C.c_int], C.c_int),
            "oracle_steady_steps": ([C.POINTER(ostc.Config), C.POINTER(ostc.Param), C.POINTER(ostc.Zone), C.c_int,
                                     C.POINTER(ostc.BcFaceC), C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
            "oracle_get_threads": ([], C.c_int),
            "oracle_chem_point_implicit": ([P, C.c_int, d, d, d, d, d, d], C.c_int),
        }
        for n, (a, r) in sig.items():
            f = getattr(L, n)
            f.argtypes = a
            f.restype = r
        _o = L
    return _o


class OracleRun:
    """Runs a Case on host copies of its blocks with the oracle."""

    def __init__(self, case):
        self.case = case
        self.blocks = [b.copy() for b in case.blocks]
        self.param, self._keep = ostc.make_param(case.scheme, case.mech)
        self.config = ostc.make_config(case.scheme)
        self.zones = (ostc.Zone * len(self.blocks))(*[b.zone() for b in self.blocks])
        self.faces = (ostc.BcFaceC * max(len(case.faces), 1))(*case.faces)
        self.nf = len(case.faces)

    def threads(self):
        return oracle().oracle_get_threads()

    def _ck(self, st, what):
        if st != 0:
            raise RuntimeError("%s -> %d" % (what, st))

    def _ifaces(self):
        ifs = list(getattr(self.case, "interfaces", []) or [])
        arr = (ostc.IfaceC * max(len(ifs), 1))(*ifs)
        oracle().oracle_set_interfaces(arr, len(ifs))

    def initialize(self):
        self._ifaces()
        self._ck(oracle().oracle_initialize(C.byref(self.config), C.byref(self.param), self.zones, len(self.blocks),
                                            self.faces, self.nf), "oracle_initialize")

    def compute_rhs(self):
        for b in range(len(self.blocks)):
            self._ck(oracle().oracle_compute_rhs(C.byref(self.param), C.byref(self.zones[b])), "oracle_compute_rhs")

    def flux_scale(self, block=0):
        """per-variable max |face flux| of one block (recomputes its dq)"""
        out = (C.c_double * self.blocks[block].n_var)()
        self._ck(oracle().oracle_flux_scale(C.byref(self.param), C.byref(self.zones[block]), out), "oracle_flux_scale")
        return np.array(out)

    def global_time_step(self):
        return oracle().oracle_global_time_step(C.byref(self.param), self.zones, len(self.blocks))

    def rk3_steps(self, n):
        self._ifaces()
        res = (C.c_double * (4 * n))()
        dts = (C.c_double * n)()
        self._ck(oracle().oracle_rk3_steps(C.byref(self.config), C.byref(self.param), self.zones, len(self.blocks),
                                           self.faces, self.nf, n, res, dts), "oracle_rk3_steps")
        return np.array(res).reshape(n, 4), np.array(dts)


    def steady_steps(self, n):
        self._ifaces()
        res = (C.c_double * (4 * n))()
        self._ck(oracle().oracle_steady_steps(C.byref(self.config), C.byref(self.param), self.zones, len(self.blocks),
                                              self.faces, self.nf, n, res), "oracle_steady_steps")
        return np.array(res).reshape(n, 4)


def chem_point_implicit(mech, T, p, Y, dt):
    """the oracle's point-implicit chemistry step of n states (numpy arrays)"""
    sch = ostc.Scheme(mix_model=ostc.MIX_FR)
    prm, keep = ostc.make_param(sch, mech)
    n = T.size
    dY = np.zeros_like(Y)
    dT = np.zeros_like(T)
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    T, p, Y, dt = [np.ascontiguousarray(a, dtype=np.float64) for a in (T, p, Y, dt)]
    st = oracle().oracle_chem_point_implicit(C.byref(prm), n, ptr(T), ptr(p), ptr(Y), ptr(dt), ptr(dY), ptr(dT))
    if st != 0:
        raise RuntimeError("oracle_chem_point_implicit -> %d" % st)
    return dY, dT


def rhs_errors(got, ref, scale, cancel=1e-2):
    """Per-variable RHS error of got vs ref (leading axis = variable):
    max|got-ref| / max(max|ref|, cancel * scale), where scale is the largest
    face flux of the variable. dq is a sum of differences of face fluxes, so
    its rounding error scales with the fluxes, not with dq itself; where
    |dq| is small against the fluxes (cancellation beyond 1/cancel) the
    denominator becomes cancel * scale."""
    out = []
    for l in range(ref.shape[0]):
        den = max(float(np.max(np.abs(ref[l]))), cancel * float(scale[l]), 1e-300)
        out.append(float(np.max(np.abs(got[l] - ref[l]))) / den)
    return out


def normwise(a, b, axis_vars=True):
    """max|a-b| / max|b| per variable (leading axis)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == 1 or not axis_vars:
        den = np.max(np.abs(b))
        return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
    out = []
    for l in range(a.shape[0]):
        den = np.max(np.abs(b[l]))
        out.append(float(np.max(np.abs(a[l] - b[l])) / (den if den > 0 else 1.0)))
    return out
