"""Python host side of the B200 RHS / RK3 path: ctypes binding of the C ABI
in include/ostc.h, block storage in the reference's DZone layout, and the
synthetic workloads.

The binding mirrors the reference's operator API (src/RK.cuh:107-161):
``Solver.compute_rhs`` is compute_source + compute_inviscid_flux +
compute_viscous_flux, ``Solver.rk3_stage`` one SSPRK3 stage, and so on. All
arithmetic runs in libostc.so (sm_100a); torch only owns device memory.
Loading fails loudly when libostc.so is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libostc.so"
MAX_SPEC = 20
MAX_REAC = 50

# status codes (include/ostc.h)
OK, ERR_INVALID_ARG, ERR_CUDA, ERR_TIMEOUT, ERR_NONPHYSICAL, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_IO = range(8)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "CUDA", 3: "TIMEOUT", 4: "NONPHYSICAL", 5: "UNSUPPORTED",
                6: "NO_DEVICE", 7: "IO"}
MIX_AIR, MIX_MIXTURE, MIX_FR = 0, 1, 2
BC_WALL, BC_SYMMETRY, BC_FARFIELD, BC_INFLOW, BC_OUTFLOW = 2, 3, 4, 5, 6
BC_SUBSONIC_INFLOW, BC_BACK_PRESSURE, BC_PERIODIC = 7, 9, 100

R_U = 8314.462618
MW_AIR = 28.9647
GAMMA_AIR = 1.4


class OstcError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__("%s failed: %s" % (what, STATUS_NAMES.get(status, status)))


# ---------------------------------------------------------------------------
# C structures (include/ostc.h)
# ---------------------------------------------------------------------------
_ZONE_PTRS = ["x", "y", "z", "jac", "metric", "wall_distance", "cv", "bv", "sv", "bv_last", "vel",
              "acoustic_speed", "mach", "mul", "thermal_conductivity", "rho_D", "gamma", "cp", "chem_src_jac",
              "mut", "turb_therm_cond", "turb_src_jac", "dq", "dq0", "dqk", "inv_spectr_rad", "visc_spectr_rad",
              "dt_local", "entropy_fix_delta", "qn"]


class Zone(C.Structure):
    _fields_ = [("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int), ("ngg", C.c_int), ("dq_ngg", C.c_int),
                ("reserved_", C.c_int)] + [(n, C.c_void_p) for n in _ZONE_PTRS]


_PARAM_INTS = ["mix_model", "turbulence", "n_var", "n_scalar", "n_spec", "n_reac", "i_turb_cv", "inviscid_scheme",
               "reconstruction", "limiter", "inviscid_type", "viscous_scheme", "rans_model", "turb_implicit",
               "compressibility_correction", "chemSrcMethod", "gradPInDiffusionFlux", "dimension"]
_PARAM_DBLS = ["entropy_fix_factor", "Pr", "Prt", "Sct", "Sc", "cfl"]
_PARAM_TABS = ["mw", "high_temp_coeff", "low_temp_coeff", "t_low", "t_mid", "t_high", "LJ_potent_inv", "vis_coeff",
               "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8", "binary_diffusivity_coeff", "kb_over_eps_jk",
               "reac_type", "stoi_f", "stoi_b", "reac_order", "A", "b", "Ea", "A2", "b2", "Ea2", "third_body_coeff",
               "troe_alpha", "troe_t3", "troe_t1", "troe_t2"]
_INT_TABS = {"reac_type", "stoi_f", "stoi_b", "reac_order"}


class Param(C.Structure):
    _fields_ = [(n, C.c_int) for n in _PARAM_INTS] + [(n, C.c_double) for n in _PARAM_DBLS] + \
               [(n, C.c_void_p) for n in _PARAM_TABS]


class BcFaceC(C.Structure):
    _fields_ = [("block", C.c_int), ("type_label", C.c_int), ("face", C.c_int), ("direction", C.c_int),
                ("range_start", C.c_int * 3), ("range_end", C.c_int * 3),
                ("density", C.c_double), ("u", C.c_double), ("v", C.c_double), ("w", C.c_double),
                ("pressure", C.c_double), ("temperature", C.c_double), ("velocity", C.c_double),
                ("mut", C.c_double), ("sv", C.c_double * (MAX_SPEC + 4)),
                ("wall_isothermal", C.c_int), ("wall_temperature", C.c_double),
                ("acoustic_speed", C.c_double), ("entropy", C.c_double), ("specific_heat_ratio", C.c_double),
                ("mw", C.c_double), ("total_pressure", C.c_double), ("total_temperature", C.c_double)]


class IfaceC(C.Structure):
    _fields_ = [("block", C.c_int), ("target", C.c_int), ("face", C.c_int), ("direction", C.c_int),
                ("range_start", C.c_int * 3), ("range_end", C.c_int * 3), ("target_start", C.c_int * 3),
                ("loop_dir", C.c_int * 3), ("target_loop_dir", C.c_int * 3), ("src_tar", C.c_int * 3),
                ("n_point", C.c_int * 3)]


class Config(C.Structure):
    _fields_ = [("steady", C.c_int), ("temporal_scheme", C.c_int), ("implicit_method", C.c_int),
                ("DPLUR_inner_step", C.c_int), ("fixed_time_step", C.c_int), ("dt", C.c_double),
                ("output_screen", C.c_int), ("compat", C.c_int), ("chem_mode", C.c_int)]


_lib = None


def lib():
    """The product library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError("libostc.so is missing at %s: run __graft_entry__.build() (no CPU fallback)" % LIB_PATH)
        L = C.CDLL(str(LIB_PATH))
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        dp, ip = C.POINTER(d), C.POINTER(i)
        sig = {
            "ostc_create": [C.POINTER(Config), C.POINTER(Param), C.POINTER(Zone), i, C.POINTER(BcFaceC), i,
                            C.POINTER(vp)],
            "ostc_destroy": [vp],
            "ostc_compute_cv_from_bv": [vp, vp],
            "ostc_compute_rhs": [vp, vp],
            "ostc_global_time_step": [vp, C.POINTER(d), vp],
            "ostc_update_cv_and_bv_rk": [vp, d, i, vp],
            "ostc_apply_boundary_conditions": [vp, i, vp],
            "ostc_data_communication": [vp, i, vp],
            "ostc_update_physical_properties": [vp, vp],
            "ostc_eliminate_k_gradient": [vp, i, vp],
            "ostc_physical_time": [vp, dp, ip],
            "ostc_set_physical_time": [vp, d, i],
            "ostc_set_monitor": [vp, i, ip, ip, ip, ip, i, ip, i, ip, i],
            "ostc_get_monitor": [vp, dp, ip],
            "ostc_set_statistics": [vp, i, i],
            "ostc_get_statistics": [vp, i, dp, dp, dp, dp, ip],
            "ostc_initialize": [vp, vp],
            "ostc_rk3_stage": [vp, i, vp],
            "ostc_rk3_steps": [vp, i, C.POINTER(d), C.POINTER(d), vp],
            "ostc_metric_from_grid": [i, i, i, i, vp, vp, vp, vp, vp],
            "ostc_get_error": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)],
            "ostc_set_tile": [vp, i, i, i],
            "ostc_get_tile": [vp, i, C.POINTER(i), C.POINTER(i)],
            "ostc_set_batching": [vp, i],
            "ostc_get_batching": [vp, C.POINTER(i)],
            "ostc_inject_wave_timeout": [vp, i],
            "ostc_launch_op": [vp, i, i, vp],
            "ostc_autotune": [vp, i, i, vp, C.POINTER(C.c_float)],
            "ostc_set_interfaces": [vp, C.POINTER(IfaceC), i],
            "ostc_step_kernel_count": [vp, i, C.POINTER(i)],
            "ostc_local_time_step": [vp, vp],
            "ostc_implicit_treatment": [vp, vp],
            "ostc_update_bv": [vp, vp],
            "ostc_steady_steps": [vp, i, C.POINTER(d), vp],
            "ostc_chem_point_implicit": [vp, i, vp, vp, vp, vp, vp, vp, vp],
            "ostc_surrogate_create": [i, C.c_ulonglong, C.POINTER(vp)],
            "ostc_surrogate_destroy": [vp],
            "ostc_surrogate_set_scaling": [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d),
                                           C.POINTER(d), C.POINTER(d), C.POINTER(d)],
            "ostc_surrogate_get_params": [vp, vp],
            "ostc_surrogate_set_params": [vp, vp],
            "ostc_surrogate_forward": [vp, vp, i, vp, vp],
            "ostc_surrogate_gradients": [vp, vp, vp, i, vp, vp, vp],
            "ostc_surrogate_forward_tc": [vp, vp, i, vp, vp],
            "ostc_surrogate_set_checks": [vp, i, i, C.POINTER(d), C.POINTER(d), d, d],
            "ostc_surrogate_inject_timeout": [vp, i],
            "ostc_write_flowfield": [vp, C.c_char_p, vp, vp, vp, vp, i, d],
            "ostc_mesh_read": [C.c_char_p, C.c_char_p, C.c_char_p, i, d, C.POINTER(vp)],
            "ostc_mesh_destroy": [vp],
            "ostc_mesh_sizes": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)],
            "ostc_mesh_block": [vp, i, C.POINTER(i), C.POINTER(i), C.POINTER(i), vp, vp, vp, vp, vp],
            "ostc_mesh_faces": [vp, vp],
            "ostc_mesh_interfaces": [vp, vp],
            "ostc_read_flowfield": [vp, C.c_char_p, vp, C.POINTER(d), C.POINTER(i)],
            "ostc_chem_surrogate": [vp, vp, i, vp, vp, vp, vp, vp, vp, C.POINTER(i), vp],
            "ostc_set_chem_surrogate": [vp, vp],
            "ostc_use_generated_chemistry": [vp, i],
            "ostc_chem_stats": [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), vp],
            "ostc_surrogate_train_step": [vp, vp, vp, i, C.c_float, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.ostc_version.restype = C.c_char_p
        L.ostc_dt_device.restype = C.c_void_p
        L.ostc_dt_device.argtypes = [vp]
        L.ostc_zone_required.restype = C.c_uint64
        L.ostc_zone_required.argtypes = [C.POINTER(Config), C.POINTER(Param)]
        _lib = L
    return _lib


def check(status: int, what: str):
    if status != OK:
        raise OstcError(status, what)


# ---------------------------------------------------------------------------
# layout helpers (ggxl ColMajor, src/gxl_lib/Array.hpp:128-194)
# ---------------------------------------------------------------------------
def plane_shape(mx, my, mz, g):
    """numpy shape of one plane: element (i,j,k) is arr[k+g, j+g, i+g]."""
    return (mz + 2 * g, my + 2 * g, mx + 2 * g)


def plane_size(mx, my, mz, g):
    return (mx + 2 * g) * (my + 2 * g) * (mz + 2 * g)


METRIC_DTYPE = np.dtype([("bias", "<i4"), ("pad", "<i4"), ("m", "<f8", (9,))])  # gxl::Matrix<real,3,3,1>


# ---------------------------------------------------------------------------
# physical tables (DParameter)
# ---------------------------------------------------------------------------
@dataclass
class Mechanism:
    """Species / reaction tables of cfd::Species and cfd::Reaction (src/ChemData.h)."""
    names: List[str]
    tables: Dict[str, np.ndarray]
    n_reac: int = 0

    @property
    def n_spec(self):
        return len(self.names)


@dataclass
class Scheme:
    mix_model: int = MIX_AIR
    inviscid_scheme: int = 3
    reconstruction: int = 2
    limiter: int = 0
    viscous_order: int = 2
    chemSrcMethod: int = 0
    gradPInDiffusionFlux: int = 0
    Pr: float = 0.72
    Prt: float = 0.9
    Sct: float = 0.9
    Sc: float = 0.9
    cfl: float = 0.5
    entropy_fix_factor: float = 0.125
    fixed_time_step: int = 0
    dt: float = 1e-6
    chem_mode: int = 0            # RK3 chemistry: 0 source in the RHS, 1 split FP64, 2 split surrogate
    rans_model: int = 0           # 0 laminar, 2 k-omega SST (air)
    compressibility_correction: int = 0  # SST: 0 none, 1 Wilcox, 2 Sarkar, 3 Zeman
    turb_implicit: int = 1        # SST, steady path: point-implicit k and omega sources (DParameter default)
    steady: int = 0               # 1: local time stepping (steady_simulation)
    implicit_method: int = 0      # steady: 0 explicit (+ EPI/DA chemistry), 1 DPLUR
    dplur_inner_step: int = 3

    @property
    def dq_ngg(self):
        # dq carries one ghost layer under DPLUR (Field.cu:213-221)
        return 1 if (self.steady and self.implicit_method == 1) else 0

    @property
    def inviscid_type(self):
        # Parameter::deduce_known_info (src/Parameter.cpp:193-198): Roe -> 2, WENO5 overrides to 1
        t = 2 if self.inviscid_scheme == 2 else 0
        if self.reconstruction in (4, 5):
            t = 1
        return t

    @property
    def ngg(self):
        return 3 if self.reconstruction == 4 else 2  # Parameter.cpp:170-180


def make_param(s: Scheme, mech: Optional[Mechanism]):
    """Returns (Param, keepalive) with host tables packed as the ABI expects."""
    p = Param()
    ns = mech.n_spec if (mech is not None and s.mix_model != MIX_AIR) else 0
    nt = 2 if s.rans_model == 2 else 0
    p.mix_model = s.mix_model
    p.turbulence = 1 if nt else 0
    p.n_spec = ns
    p.n_scalar = ns + nt
    p.n_var = 5 + ns + nt
    p.n_reac = mech.n_reac if (mech is not None and s.mix_model == MIX_FR) else 0
    p.i_turb_cv = 5 + ns
    p.inviscid_scheme = s.inviscid_scheme
    p.reconstruction = s.reconstruction
    p.limiter = s.limiter
    p.inviscid_type = s.inviscid_type
    p.viscous_scheme = s.viscous_order
    p.rans_model = s.rans_model
    p.turb_implicit = s.turb_implicit if nt else 0
    p.compressibility_correction = s.compressibility_correction if nt else 0
    p.chemSrcMethod = s.chemSrcMethod
    p.gradPInDiffusionFlux = s.gradPInDiffusionFlux
    p.dimension = 3
    for n in _PARAM_DBLS:
        setattr(p, n, getattr(s, n))
    keep = []
    if ns:
        for n in _PARAM_TABS:
            if n not in mech.tables:
                continue
            arr = np.ascontiguousarray(mech.tables[n], dtype=np.int32 if n in _INT_TABS else np.float64)
            keep.append(arr)
            setattr(p, n, arr.ctypes.data)
    return p, keep


def make_config(s: Scheme, output_screen: int = 1) -> Config:
    c = Config()
    c.steady = s.steady
    c.temporal_scheme = 3
    c.implicit_method = s.implicit_method
    c.DPLUR_inner_step = s.dplur_inner_step
    c.fixed_time_step = s.fixed_time_step
    c.dt = s.dt
    c.output_screen = output_screen
    c.compat = 1
    c.chem_mode = s.chem_mode
    return c


# ---------------------------------------------------------------------------
# block storage
# ---------------------------------------------------------------------------
@dataclass
class HostBlock:
    """One block in the reference layout, host (numpy) side."""
    mx: int
    my: int
    mz: int
    ngg: int
    n_var: int
    n_spec: int
    arrays: Dict[str, np.ndarray] = field(default_factory=dict)
    dq_ngg: int = 0
    n_turb: int = 0  # turbulence scalars after the species in sv (2 with SST)

    def plane(self, g=None):
        return plane_shape(self.mx, self.my, self.mz, self.ngg if g is None else g)

    @staticmethod
    def specs(mx, my, mz, ngg, n_var, n_spec, dq_ngg=0, n_turb=0):
        """name -> (shape, dtype) of every array of a block (Field::setup_device_memory)."""
        P = plane_shape(mx, my, mz, ngg)
        I = plane_shape(mx, my, mz, 0)
        Q = plane_shape(mx, my, mz, dq_ngg)
        f8 = np.float64
        sp = {"bv": ((6,) + P, f8), "sv": ((n_spec + n_turb,) + P, f8), "cv": ((n_var,) + P, f8),
              "qn": ((n_var,) + P, f8), "dq": ((n_var,) + Q, f8), "jac": (P, f8), "metric": (P, METRIC_DTYPE)}
        for n in ("vel", "acoustic_speed", "mach", "mul", "thermal_conductivity"):
            sp[n] = (P, f8)
        if n_spec:
            sp["rho_D"] = ((n_spec,) + P, f8)
            sp["gamma"] = (P, f8)
            sp["cp"] = (P, f8)
        if n_turb:
            for n in ("mut", "turb_therm_cond", "wall_distance"):
                sp[n] = (P, f8)
            sp["turb_src_jac"] = ((2,) + I, f8)
        sp["dt_local"] = (I, f8)
        sp["bv_last"] = ((4,) + I, f8)
        return sp

    INPUTS = ("bv", "sv", "jac", "metric", "wall_distance")

    @staticmethod
    def allocate(mx, my, mz, ngg, n_var, n_spec, full=True, dq_ngg=0, n_turb=0) -> "HostBlock":
        """full=False holds only the inputs (bv, sv, jac, metric, wall
        distance); the device block creates the rest zero-filled."""
        b = HostBlock(mx, my, mz, ngg, n_var, n_spec, dq_ngg=dq_ngg, n_turb=n_turb)
        for n, (shape, dt) in HostBlock.specs(mx, my, mz, ngg, n_var, n_spec, dq_ngg, n_turb).items():
            if full or n in HostBlock.INPUTS:
                b.arrays[n] = np.zeros(shape, dtype=dt)
        return b

    def complete(self) -> "HostBlock":
        """a full copy (all arrays) for the oracle"""
        b = HostBlock.allocate(self.mx, self.my, self.mz, self.ngg, self.n_var, self.n_spec, full=True,
                               dq_ngg=self.dq_ngg, n_turb=self.n_turb)
        for n, v in self.arrays.items():
            b.arrays[n][...] = v
        return b

    def copy(self) -> "HostBlock":
        return self.complete()

    def zone(self) -> Zone:
        z = Zone()
        z.mx, z.my, z.mz, z.ngg, z.dq_ngg = self.mx, self.my, self.mz, self.ngg, self.dq_ngg
        for n, v in self.arrays.items():
            if v.size:
                setattr(z, n, v.ctypes.data)
        return z


class DeviceBlock:
    """One block on the GPU (torch-owned memory), same layout as HostBlock."""

    def __init__(self, host: HostBlock, device="cuda"):
        import torch

        self.host_shape = host
        self.mx, self.my, self.mz, self.ngg = host.mx, host.my, host.mz, host.ngg
        self.dq_ngg = host.dq_ngg
        self.specs = HostBlock.specs(host.mx, host.my, host.mz, host.ngg, host.n_var, host.n_spec, host.dq_ngg,
                                     host.n_turb)
        self.t = {}
        for n, (shape, dt) in self.specs.items():
            if n == "metric":
                nbytes = int(np.prod(shape)) * METRIC_DTYPE.itemsize
                self.t[n] = torch.zeros(nbytes, dtype=torch.uint8, device=device)
            else:
                self.t[n] = torch.zeros(shape, dtype=torch.float64, device=device)
        self.upload_inputs(host)

    def upload_inputs(self, host: HostBlock, names=None):
        import torch

        for n in names or host.arrays.keys():
            v = host.arrays[n]
            if n == "metric":
                self.t[n].copy_(torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).reshape(-1)))
            else:
                self.t[n].copy_(torch.from_numpy(np.ascontiguousarray(v)))

    def zone(self) -> Zone:
        z = Zone()
        z.mx, z.my, z.mz, z.ngg, z.dq_ngg = self.mx, self.my, self.mz, self.ngg, self.dq_ngg
        for n, v in self.t.items():
            if v.numel():
                setattr(z, n, v.data_ptr())
        return z

    def download(self, name) -> np.ndarray:
        v = self.t[name].cpu().numpy()
        if name == "metric":
            return v.view(METRIC_DTYPE).reshape(self.specs["metric"][0])
        return v

    def upload(self, name, arr: np.ndarray):
        import torch

        self.t[name].copy_(torch.from_numpy(np.ascontiguousarray(arr)))


# ---------------------------------------------------------------------------
# boundary faces
# ---------------------------------------------------------------------------
def bc_face(block: int, label: int, face: int, direction: int, ext, ngg, state: Optional[dict] = None) -> BcFaceC:
    """A face of one block after Boundary::register_boundary (src/Mesh.cpp:14-32):
    the tangential ranges are widened by ngg; wall faces are trimmed back by
    ngg as DBoundCond::initialize_bc_on_GPU does (src/BoundCond.cu:369-387)."""
    f = BcFaceC()
    f.block, f.type_label, f.face, f.direction = block, label, face, direction
    trim = ngg if label == BC_WALL else 0
    for d in range(3):
        if d == face:
            v = 0 if direction < 0 else ext[d] - 1
            f.range_start[d] = v
            f.range_end[d] = v
        else:
            f.range_start[d] = -ngg + trim
            f.range_end[d] = ext[d] - 1 + ngg - trim
    if state:
        for k in ("density", "u", "v", "w", "pressure", "temperature", "velocity", "mut", "acoustic_speed", "entropy",
                  "specific_heat_ratio", "mw", "total_pressure", "total_temperature", "wall_temperature"):
            setattr(f, k, float(state.get(k, 0.0)))
        f.wall_isothermal = int(state.get("wall_isothermal", 0))
        for l, y in enumerate(state.get("sv", [])):
            f.sv[l] = float(y)
    return f


def farfield_state(mach, T, p, direction=(1.0, 0.0, 0.0), mech: Optional[Mechanism] = None, Y=None):
    """The state of cfd::FarField for (mach, pressure, temperature) input
    (src/BoundCond.cpp:184-266): sound speed, velocity, density, entropy."""
    mw, gamma, sv = MW_AIR, GAMMA_AIR, []
    if mech is not None:
        Y = np.asarray(Y, dtype=float)
        t = mech.tables
        mw = 1.0 / float(np.sum(Y / t["mw"]))
        cp_i = np.empty(len(Y))
        for i in range(len(Y)):
            if T < t["t_low"][i]:
                c, tt = t["low_temp_coeff"][i], t["t_low"][i]
            else:
                c, tt = (t["low_temp_coeff"][i] if T < t["t_mid"][i] else t["high_temp_coeff"][i]), T
            cp_i[i] = (c[0] + c[1] * tt + c[2] * tt ** 2 + c[3] * tt ** 3 + c[4] * tt ** 4) * R_U / t["mw"][i]
        cp = float(np.sum(Y * cp_i))
        cv = float(np.sum(Y * (cp_i - R_U / t["mw"])))
        gamma = cp / cv
        sv = list(Y)
    a = math.sqrt(gamma * R_U / mw * T)
    vel = mach * a
    rho = p * mw / (R_U * T)
    return dict(density=rho, u=direction[0] * vel, v=direction[1] * vel, w=direction[2] * vel, pressure=p,
                temperature=T, velocity=vel, acoustic_speed=a, entropy=p / rho ** gamma, specific_heat_ratio=gamma,
                mw=mw, sv=sv)


# ---------------------------------------------------------------------------
# the solver (one ostc_ctx)
# ---------------------------------------------------------------------------
class Solver:
    def __init__(self, scheme: Scheme, mech: Optional[Mechanism], blocks: List[DeviceBlock], faces: List[BcFaceC],
                 output_screen: int = 1, interfaces: Optional[List["IfaceC"]] = None):
        import torch

        self.scheme = scheme
        self.mech = mech
        self.blocks = blocks
        self.param, self._keep = make_param(scheme, mech)
        self.config = make_config(scheme, output_screen)
        zones = (Zone * len(blocks))(*[b.zone() for b in blocks])
        self._zones = zones
        fa = (BcFaceC * max(len(faces), 1))(*faces)
        self._faces = fa
        ctx = C.c_void_p()
        check(lib().ostc_create(C.byref(self.config), C.byref(self.param), zones, len(blocks), fa, len(faces),
                                C.byref(ctx)), "ostc_create")
        self.ctx = ctx
        self.stream = torch.cuda.current_stream().cuda_stream
        if interfaces:
            ia = (IfaceC * len(interfaces))(*interfaces)
            self._ifaces = ia
            check(lib().ostc_set_interfaces(self.ctx, ia, len(interfaces)), "ostc_set_interfaces")

    def close(self):
        if self.ctx:
            lib().ostc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self):
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def initialize(self):
        check(lib().ostc_initialize(self.ctx, self._s()), "ostc_initialize")

    def compute_rhs(self):
        check(lib().ostc_compute_rhs(self.ctx, self._s()), "ostc_compute_rhs")

    def compute_cv_from_bv(self):
        check(lib().ostc_compute_cv_from_bv(self.ctx, self._s()), "ostc_compute_cv_from_bv")

    def global_time_step(self) -> float:
        dt = C.c_double()
        check(lib().ostc_global_time_step(self.ctx, C.byref(dt), self._s()), "ostc_global_time_step")
        return dt.value

    def update_cv_and_bv_rk(self, dt: float, rk: int):
        check(lib().ostc_update_cv_and_bv_rk(self.ctx, dt, rk, self._s()), "ostc_update_cv_and_bv_rk")

    def apply_boundary_conditions(self, with_cv: bool):
        check(lib().ostc_apply_boundary_conditions(self.ctx, int(with_cv), self._s()), "ostc_apply_bc")

    def update_physical_properties(self):
        check(lib().ostc_update_physical_properties(self.ctx, self._s()), "ostc_update_physical_properties")

    def eliminate_k_gradient(self, with_cv: bool):
        """2-D blocks: the k ghost planes take the plane k = 0 (a no-op in 3-D)"""
        check(lib().ostc_eliminate_k_gradient(self.ctx, int(with_cv), self._s()), "ostc_eliminate_k_gradient")

    def physical_time(self):
        """(physical time, step count) of the RK3 loop since initialize"""
        t, n = C.c_double(), C.c_int()
        check(lib().ostc_physical_time(self.ctx, C.byref(t), C.byref(n)), "ostc_physical_time")
        return t.value, n.value

    def set_physical_time(self, time: float, step: int):
        """continue a restarted run from (time, step) (call after initialize)"""
        check(lib().ostc_set_physical_time(self.ctx, float(time), int(step)), "ostc_set_physical_time")

    def set_monitor(self, points, bv_labels=(0, 1, 2, 3, 4, 5), sv_labels=(), capacity=64):
        """monitor points [(block, i, j, k), ...]; [] removes the monitor"""
        n = len(points)
        cols = [np.ascontiguousarray([p[c] for p in points], dtype=np.int32) for c in range(4)] if n else [
            np.zeros(1, np.int32)] * 4
        bl = np.ascontiguousarray(bv_labels, dtype=np.int32)
        sl = np.ascontiguousarray(sv_labels, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        check(lib().ostc_set_monitor(self.ctx, n, *[c.ctypes.data_as(ip) for c in cols], len(bl),
                                     bl.ctypes.data_as(ip) if len(bl) else None, len(sl),
                                     sl.ctypes.data_as(ip) if len(sl) else None, capacity), "ostc_set_monitor")
        self._monitor = (n, len(bl) + len(sl) + 1, capacity)

    def get_monitor(self):
        """records since the last read: array [point][step][bv labels, sv labels, time]"""
        n, nv, cap = getattr(self, "_monitor", (0, 0, 0))
        out = np.zeros((max(n, 1), cap, nv))
        rec = C.c_int()
        check(lib().ostc_get_monitor(self.ctx, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(rec)),
              "ostc_get_monitor")
        return out[:n, :rec.value]

    def _names(self):
        names = list(self.mech.names) if (self.mech is not None and self.param.n_spec > 0) else []
        arr = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
        return arr if names else None

    def write_flowfield(self, path, coords, ngg_out=0, solution_time=0.0):
        """the reference's restart / output file (ostc_write_flowfield);
        coords: per block (x, y, z) host arrays with the block's ghost layers"""
        keep = [np.ascontiguousarray(a, dtype=np.float64) for xyz in coords for a in xyz]
        ptrs = [(C.c_void_p * len(coords))(*[keep[3 * b + c].ctypes.data for b in range(len(coords))])
                for c in range(3)]
        check(lib().ostc_write_flowfield(self.ctx, str(path).encode(), *ptrs, self._names(), ngg_out,
                                         float(solution_time)), "ostc_write_flowfield")

    def read_flowfield(self, path):
        """fills bv / sv from such a file; returns (solution_time, found bits)"""
        t, f = C.c_double(), C.c_int()
        check(lib().ostc_read_flowfield(self.ctx, str(path).encode(), self._names(), C.byref(t), C.byref(f)),
              "ostc_read_flowfield")
        return t.value, f.value

    def get_error(self):
        """the context's last status and, for OSTC_ERR_NONPHYSICAL, the first
        failing cell: (status, cuda_error, block, i, j, k)"""
        v = [C.c_int() for _ in range(5)]
        st = lib().ostc_get_error(self.ctx, *[C.byref(x) for x in v])
        return (st,) + tuple(x.value for x in v)

    def set_statistics(self, on=True, start_step=0):
        check(lib().ostc_set_statistics(self.ctx, int(bool(on)), start_step), "ostc_set_statistics")

    def get_statistics(self, block=0):
        """per-cell sums of one block (interior): sum12 [12], sum34 [12], sum_rs [3], sum_yk [n_spec], count"""
        b = self.blocks[block]
        shape = (b.mz, b.my, b.mx)
        ns = self.param.n_spec
        out = {"sum12": np.zeros((12,) + shape), "sum34": np.zeros((12,) + shape), "sum_rs": np.zeros((3,) + shape),
               "sum_yk": np.zeros((max(ns, 1),) + shape)}
        dp = C.POINTER(C.c_double)
        cnt = C.c_int()
        check(lib().ostc_get_statistics(self.ctx, block, *[out[k].ctypes.data_as(dp) for k in
                                                           ("sum12", "sum34", "sum_rs", "sum_yk")], C.byref(cnt)),
              "ostc_get_statistics")
        out["sum_yk"] = out["sum_yk"][:ns]
        out["count"] = cnt.value
        return out

    def rk3_stage(self, rk: int):
        check(lib().ostc_rk3_stage(self.ctx, rk, self._s()), "ostc_rk3_stage")

    def rk3_steps(self, n: int, history: bool = False):
        if history:
            res = (C.c_double * (4 * n))()
            dts = (C.c_double * n)()
            check(lib().ostc_rk3_steps(self.ctx, n, res, dts, self._s()), "ostc_rk3_steps")
            return np.array(res).reshape(n, 4), np.array(dts)
        check(lib().ostc_rk3_steps(self.ctx, n, None, None, self._s()), "ostc_rk3_steps")
        return None

    # steady path (SteadySim.cuh:15-137)
    def local_time_step(self):
        check(lib().ostc_local_time_step(self.ctx, self._s()), "ostc_local_time_step")

    def implicit_treatment(self):
        check(lib().ostc_implicit_treatment(self.ctx, self._s()), "ostc_implicit_treatment")

    def update_bv(self):
        check(lib().ostc_update_bv(self.ctx, self._s()), "ostc_update_bv")

    def steady_steps(self, n: int, history: bool = False):
        if history:
            res = (C.c_double * (4 * n))()
            check(lib().ostc_steady_steps(self.ctx, n, res, self._s()), "ostc_steady_steps")
            return np.array(res).reshape(n, 4)
        check(lib().ostc_steady_steps(self.ctx, n, None, self._s()), "ostc_steady_steps")
        return None

    def use_generated_chemistry(self, on: bool):
        check(lib().ostc_use_generated_chemistry(self.ctx, int(on)), "ostc_use_generated_chemistry")

    def set_chem_surrogate(self, sur):
        """the surrogate of chem_mode 2 (kept alive by this solver)"""
        check(lib().ostc_set_chem_surrogate(self.ctx, sur.h), "ostc_set_chem_surrogate")
        self._sur = sur

    def chem_stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        check(lib().ostc_chem_stats(self.ctx, C.byref(a), C.byref(b), self._s()), "ostc_chem_stats")
        return a.value, b.value

    def chem_surrogate(self, sur, T, p, Y, dt):
        """learned chemistry step with FP64 fallback (torch CUDA tensors as for
        chem_point_implicit); returns (dY, dT, number of states redone)."""
        import torch

        n = T.numel()
        dY = torch.empty_like(Y)
        dT = torch.empty_like(T)
        nfb = C.c_int()
        check(lib().ostc_chem_surrogate(self.ctx, sur.h, n, T.data_ptr(), p.data_ptr(), Y.data_ptr(), dt.data_ptr(),
                                        dY.data_ptr(), dT.data_ptr(), C.byref(nfb), self._s()), "ostc_chem_surrogate")
        return dY, dT, nfb.value

    def chem_point_implicit(self, T, p, Y, dt):
        """FP64 point-implicit chemistry step of each state (torch CUDA tensors:
        T, p, dt [n]; Y [n_spec, n]); returns (dY [n_spec, n], dT [n])."""
        import torch

        n = T.numel()
        dY = torch.empty_like(Y)
        dT = torch.empty_like(T)
        check(lib().ostc_chem_point_implicit(self.ctx, n, T.data_ptr(), p.data_ptr(), Y.data_ptr(), dt.data_ptr(),
                                             dY.data_ptr(), dT.data_ptr(), self._s()), "ostc_chem_point_implicit")
        return dY, dT

    OP_FLUX, OP_SOURCE, OP_PROPERTIES, OP_UPDATE, OP_DT, OP_BC = range(6)

    def launch_op(self, op, arg=0):
        check(lib().ostc_launch_op(self.ctx, op, arg, self._s()), "ostc_launch_op")

    def step_kernel_count(self, with_hist=False):
        n = C.c_int()
        check(lib().ostc_step_kernel_count(self.ctx, int(with_hist), C.byref(n)), "ostc_step_kernel_count")
        return n.value

    def set_batching(self, on: bool):
        """one persistent tile-table launch per kernel over all blocks, and
        one launch per call for the boundary faces and for the interfaces
        (True), or one launch per block and face (False)"""
        check(lib().ostc_set_batching(self.ctx, int(bool(on))), "ostc_set_batching")

    def inject_wave_timeout(self, on: bool):
        """diagnostic: make the grid barriers of the batched boundary-face and
        interface launches run out (calls with histories then return
        OSTC_ERR_TIMEOUT)"""
        check(lib().ostc_inject_wave_timeout(self.ctx, 1 if on else 0), "ostc_inject_wave_timeout")

    def batching(self) -> bool:
        v = C.c_int()
        check(lib().ostc_get_batching(self.ctx, C.byref(v)), "ostc_get_batching")
        return bool(v.value)

    def set_tile(self, d, rows, chunks):
        check(lib().ostc_set_tile(self.ctx, d, rows, chunks), "ostc_set_tile")

    def get_tile(self, d):
        r, c = C.c_int(), C.c_int()
        check(lib().ostc_get_tile(self.ctx, d, C.byref(r), C.byref(c)), "ostc_get_tile")
        return r.value, c.value

    def tiles(self):
        """the six tile settings: fused/inviscid flux of x, y, z, then the
        separate viscous flux of x, y, z ((0, 0) = fused)"""
        return [self.get_tile(d) for d in range(6)]

    def set_tiles(self, tiles):
        for d, (r, c) in enumerate(tiles or []):
            self.set_tile(d, r, c)

    def _time_flux(self, arg, warmup, reps):
        """device ms of one flux launch (op argument arg), or None when the
        tile setting cannot run for this scheme (a staged kernel for AWENO,
        or a tile larger than a CTA's shared memory)"""
        import torch

        try:
            self.launch_op(self.OP_FLUX, arg)
        except OstcError:
            return None
        for _ in range(warmup):
            self.launch_op(self.OP_FLUX, arg)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            self.launch_op(self.OP_FLUX, arg)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def autotune(self, warmup: int = 1, reps: int = 3, verbose: bool = False):
        """Pick per-direction flux tile shapes (rows, chunks, register budget,
        staged or not) with the library's autotuner (ostc_autotune), which
        times each flux kernel with CUDA events on the launching stream; for a
        viscous flow the fused kernel competes with the pair of separate
        inviscid and viscous kernels. Only dq is written, so the state is left
        as it was. Returns {direction: (ms, tile, viscous tile)}."""
        ms = (C.c_float * 3)()
        check(lib().ostc_autotune(self.ctx, warmup, reps, self._s(), ms), "ostc_autotune")
        best = {d: (float(ms[d]), self.get_tile(d), self.get_tile(d + 3)) for d in range(3)}
        if verbose:
            for d in range(3):
                print("dir", d, "chosen", best[d])
        return best


# ---------------------------------------------------------------------------
# synthetic workloads
# ---------------------------------------------------------------------------
def grid_coordinates(mx, my, mz, ng, dx, warp=0.02, periodic_k=True):
    """Node coordinates with ng ghost layers: x = i dx plus a 2% sinusoidal
    curvilinear warp, periodic in k with period mz*dx (nodes k = 0..mz-1
    are distinct), analytic in the ghost layers. mz == 1 is a 2-D grid: the
    warp stays in the (x, y) plane and the k ghost nodes sit at z = k, as
    the reference's grid reader places them (src/Mesh.cpp:840-854)."""
    i = np.arange(-ng, mx + ng, dtype=np.float64)
    j = np.arange(-ng, my + ng, dtype=np.float64)
    k = np.arange(-ng, mz + ng, dtype=np.float64)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    Lx, Ly, Lz = (mx - 1) * dx, (my - 1) * dx, mz * dx
    x0, y0, z0 = I * dx, J * dx, K * dx
    if mz == 1:
        sx, sy = np.sin(2 * np.pi * x0 / Lx), np.sin(2 * np.pi * y0 / Ly)
        return x0 + warp * dx * sy, y0 + warp * dx * sx, K.copy()
    sx, sy, sz = np.sin(2 * np.pi * x0 / Lx), np.sin(2 * np.pi * y0 / Ly), np.sin(2 * np.pi * z0 / Lz)
    x = x0 + warp * dx * sy * sz
    y = y0 + warp * dx * sx * sz
    z = z0 + warp * dx * sx * sy
    return x, y, z


_metric_provider = None


def set_metric_provider(fn):
    """Route the synthetic workloads' geometry through fn(mx, my, mz, ngg, x,
    y, z) -> (jac, metric) instead of ostc_metric_from_grid (None restores
    the library's helper). For callers that build the same workloads without
    loading the library, such as a CPU baseline."""
    global _metric_provider
    _metric_provider = fn


def fill_metric(block: HostBlock, x, y, z):
    if _metric_provider is not None:
        jac, met = _metric_provider(block.mx, block.my, block.mz, block.ngg, x, y, z)
        block.arrays["jac"][...] = jac
        block.arrays["metric"][...] = met.view(block.arrays["metric"].dtype)
        return
    check(lib().ostc_metric_from_grid(block.mx, block.my, block.mz, block.ngg, x.ctypes.data, y.ctypes.data,
                                      z.ctypes.data, block.arrays["jac"].ctypes.data,
                                      block.arrays["metric"].ctypes.data), "ostc_metric_from_grid")


@dataclass
class Case:
    name: str
    scheme: Scheme
    mech: Optional[Mechanism]
    blocks: List[HostBlock]
    faces: List[BcFaceC]
    steps: int
    interfaces: List["IfaceC"] = field(default_factory=list)

    def solver(self, **kw):
        """A Solver on fresh device copies of the blocks."""
        blocks = [DeviceBlock(b) for b in self.blocks]
        return Solver(self.scheme, self.mech, blocks, self.faces, interfaces=self.interfaces, **kw), blocks

    @property
    def cells(self):
        return sum(b.mx * b.my * b.mz for b in self.blocks)


def air_state(mach, T, p):
    a = math.sqrt(GAMMA_AIR * R_U / MW_AIR * T)
    rho = p * MW_AIR / (R_U * T)
    return dict(density=rho, u=mach * a, v=0.0, w=0.0, pressure=p, temperature=T, velocity=mach * a, mut=0.0)


def case_vortex(mx=128, my=128, mz=8, dx=1e-3, k_bc="periodic", steps=100, fixed_dt=None, reconstruction=4,
                inviscid_scheme=2) -> Case:
    """The single-species air workload: a Mach 2 stream (T = 300 K,
    p = 101325 Pa) along +x with an isentropic vortex (strength 0.3 U_inf,
    radius 5 dx) at the domain centre; AWENO-5 with the Roe tag (which runs
    AUSM+ in the reference, quirk A1), laminar Sutherland viscosity, RK3 at
    CFL 0.5. Supersonic inlet at i-min, supersonic outlet at i-max, symmetry
    on the j faces, periodic in k (k_bc="periodic") or symmetry in k
    (k_bc="symmetry", a configuration the reference itself can run).
    Other reconstruction / flux tags give the other air schemes (2 + 2 is the
    Roe flux-difference splitting with MUSCL)."""
    s = Scheme(mix_model=MIX_AIR, inviscid_scheme=inviscid_scheme, reconstruction=reconstruction, viscous_order=2,
               cfl=0.5)
    if fixed_dt:
        s.fixed_time_step, s.dt = 1, fixed_dt
    ng = s.ngg
    b = HostBlock.allocate(mx, my, mz, ng, 5, 0)
    x, y, z = grid_coordinates(mx, my, mz, ng + 1, dx, periodic_k=True)
    fill_metric(b, x, y, z)
    inf = air_state(2.0, 300.0, 101325.0)
    # state on all points incl. ghosts (coordinates with ng layers)
    xs, ys = x[1:-1, 1:-1, 1:-1], y[1:-1, 1:-1, 1:-1]
    xc, yc = (mx // 2) * dx, (my // 2) * dx
    R, beta = 5 * dx, 0.3
    U = inf["u"]
    r2 = ((xs - xc) ** 2 + (ys - yc) ** 2) / R ** 2
    ex = np.exp(0.5 * (1 - r2))
    Rg = R_U / MW_AIR
    T = 300.0 - (GAMMA_AIR - 1) / (2 * GAMMA_AIR) * (beta * U) ** 2 / Rg * ex ** 2
    rho = inf["density"] * (T / 300.0) ** (1 / (GAMMA_AIR - 1))
    bv = b.arrays["bv"]
    bv[0] = rho
    bv[1] = U - beta * U * (ys - yc) / R * ex
    bv[2] = beta * U * (xs - xc) / R * ex
    bv[3] = 0.0
    bv[4] = rho * Rg * T
    bv[5] = T
    ext = (mx, my, mz)
    faces = [bc_face(0, BC_INFLOW, 0, -1, ext, ng, inf), bc_face(0, BC_OUTFLOW, 0, 1, ext, ng),
             bc_face(0, BC_SYMMETRY, 1, -1, ext, ng), bc_face(0, BC_SYMMETRY, 1, 1, ext, ng)]
    if mz == 1:  # 2-D: no k faces (the k ghost planes copy k = 0)
        pass
    elif k_bc == "periodic":
        faces += [bc_face(0, BC_PERIODIC, 2, -1, ext, ng), bc_face(0, BC_PERIODIC, 2, 1, ext, ng)]
    else:
        faces += [bc_face(0, BC_SYMMETRY, 2, -1, ext, ng), bc_face(0, BC_SYMMETRY, 2, 1, ext, ng)]
    return Case("vortex_air_%dx%dx%d" % (mx, my, mz), s, None, [b], faces, steps)


def case_bc_box(kind="wall_farfield", mx=40, my=32, mz=10, dx=1e-3) -> Case:
    """Air box exercising the wall, far-field, back-pressure and subsonic
    inflow conditions: a Mach 0.5 stream (300 K, 1 atm) with the vortex of
    case_vortex, MUSCL + AUSM+, laminar; symmetry in k (runnable by the
    reference build).
    kind="wall_farfield": far field at i-min and j-max, back pressure at
    i-max, isothermal 300 K wall at j-min.
    kind="subsonic": subsonic inflow (total conditions of the stream) at i-min,
    back pressure at i-max, adiabatic wall at j-min, symmetry at j-max."""
    c = case_vortex(mx, my, mz, dx, k_bc="symmetry", reconstruction=2, inviscid_scheme=3)
    b = c.blocks[0]
    ng = b.ngg
    ff = farfield_state(0.5, 300.0, 101325.0)
    # re-scale the vortex field to the Mach 0.5 stream
    bv = b.arrays["bv"]
    scale = ff["u"] / air_state(2.0, 300.0, 101325.0)["u"]
    bv[1] *= scale
    bv[2] *= scale
    Rg = R_U / MW_AIR
    bv[5] = 300.0 - (300.0 - bv[5]) * scale ** 2
    bv[0] = ff["density"] * (bv[5] / 300.0) ** (1 / (GAMMA_AIR - 1))
    bv[4] = bv[0] * Rg * bv[5]
    ext = (mx, my, mz)
    wall = dict(wall_isothermal=1, wall_temperature=300.0)
    bp = dict(pressure=101325.0)
    if kind == "wall_farfield":
        faces = [bc_face(0, BC_FARFIELD, 0, -1, ext, ng, ff), bc_face(0, BC_BACK_PRESSURE, 0, 1, ext, ng, bp),
                 bc_face(0, BC_WALL, 1, -1, ext, ng, wall), bc_face(0, BC_FARFIELD, 1, 1, ext, ng, ff)]
    else:
        M = 0.5
        tot = dict(total_pressure=101325.0 * (1 + 0.2 * M * M) ** 3.5, total_temperature=300.0 * (1 + 0.2 * M * M),
                   u=1.0, v=0.0, w=0.0)
        faces = [bc_face(0, BC_SUBSONIC_INFLOW, 0, -1, ext, ng, tot), bc_face(0, BC_BACK_PRESSURE, 0, 1, ext, ng, bp),
                 bc_face(0, BC_WALL, 1, -1, ext, ng, dict(wall_isothermal=0)),
                 bc_face(0, BC_SYMMETRY, 1, 1, ext, ng)]
    if mz > 1:
        faces += [bc_face(0, BC_SYMMETRY, 2, -1, ext, ng), bc_face(0, BC_SYMMETRY, 2, 1, ext, ng)]
    c.faces = faces
    c.name = "bc_box_%s_%dx%dx%d" % (kind, mx, my, mz)
    return c


def iface_aligned(block, target, face, direction, ext_self, ext_tar, ngg) -> IfaceC:
    """The registered cfd::InnerFace (src/Mesh.cpp:34-178) of two blocks whose
    axes are aligned and whose coincident planes are `face`-max of one and
    `face`-min of the other; tangential ranges cover the interior only."""
    f = IfaceC()
    f.block, f.target, f.face, f.direction = block, target, face, direction
    for d in range(3):
        f.loop_dir[d] = 1
        f.target_loop_dir[d] = 1
        f.src_tar[d] = d
        if d == face:
            if direction > 0:
                f.range_start[d], f.range_end[d] = ext_self[d] - 1, ext_self[d] - 1 + ngg
                f.target_start[d] = 0
            else:
                f.range_start[d], f.range_end[d] = -ngg, 0
                f.target_start[d] = ext_tar[d] - 1 - ngg
            f.n_point[d] = ngg + 1
        else:
            f.range_start[d], f.range_end[d] = 0, ext_self[d] - 1
            f.target_start[d] = 0
            f.n_point[d] = ext_self[d]
    return f


def case_multiblock(nx=(20, 17, 13), ny=(15, 19), mz=8, dx=1e-3, reconstruction=4, inviscid_scheme=2) -> Case:
    """The air vortex of case_vortex on a grid split into len(nx) x len(ny)
    blocks of uneven sizes that share their face planes (1-to-1 interfaces,
    averaged on the shared plane, quirk A10); inflow / outflow in i,
    symmetry in j and k, so the reference build can run it."""
    s = Scheme(mix_model=MIX_AIR, inviscid_scheme=inviscid_scheme, reconstruction=reconstruction, viscous_order=2,
               cfl=0.5)
    ng = s.ngg
    NX = sum(nx) - (len(nx) - 1)
    NY = sum(ny) - (len(ny) - 1)
    xg, yg, zg = grid_coordinates(NX, NY, mz, ng + 1, dx, periodic_k=True)
    inf = air_state(2.0, 300.0, 101325.0)
    xs, ys = xg[1:-1, 1:-1, 1:-1], yg[1:-1, 1:-1, 1:-1]
    xc, yc = (NX // 2) * dx, (NY // 2) * dx
    R, beta, U = 5 * dx, 0.3, inf["u"]
    r2 = ((xs - xc) ** 2 + (ys - yc) ** 2) / R ** 2
    ex = np.exp(0.5 * (1 - r2))
    Rg = R_U / MW_AIR
    T = 300.0 - (GAMMA_AIR - 1) / (2 * GAMMA_AIR) * (beta * U) ** 2 / Rg * ex ** 2
    rho = inf["density"] * (T / 300.0) ** (1 / (GAMMA_AIR - 1))
    gbv = np.stack([rho, U - beta * U * (ys - yc) / R * ex, beta * U * (xs - xc) / R * ex, 0 * rho, rho * Rg * T, T])
    blocks, faces, ifaces, ids = [], [], [], {}
    ox = np.cumsum([0] + [n - 1 for n in nx])
    oy = np.cumsum([0] + [n - 1 for n in ny])
    for bj, my in enumerate(ny):
        for bi, mx in enumerate(nx):
            b = HostBlock.allocate(mx, my, mz, ng, 5, 0)
            i0, j0 = ox[bi], oy[bj]
            sl = (slice(None), slice(j0, j0 + my + 2 * ng + 2), slice(i0, i0 + mx + 2 * ng + 2))
            fill_metric(b, np.ascontiguousarray(xg[sl]), np.ascontiguousarray(yg[sl]), np.ascontiguousarray(zg[sl]))
            b.arrays["bv"][...] = gbv[:, :, j0:j0 + my + 2 * ng, i0:i0 + mx + 2 * ng]
            ids[(bi, bj)] = len(blocks)
            blocks.append(b)
    for (bi, bj), q in ids.items():
        ext = (nx[bi], ny[bj], mz)
        if bi == 0:
            faces.append(bc_face(q, BC_INFLOW, 0, -1, ext, ng, inf))
        else:
            t = ids[(bi - 1, bj)]
            ifaces.append(iface_aligned(q, t, 0, -1, ext, (nx[bi - 1], ny[bj], mz), ng))
        if bi == len(nx) - 1:
            faces.append(bc_face(q, BC_OUTFLOW, 0, 1, ext, ng))
        else:
            t = ids[(bi + 1, bj)]
            ifaces.append(iface_aligned(q, t, 0, 1, ext, (nx[bi + 1], ny[bj], mz), ng))
        if bj == 0:
            faces.append(bc_face(q, BC_SYMMETRY, 1, -1, ext, ng))
        else:
            t = ids[(bi, bj - 1)]
            ifaces.append(iface_aligned(q, t, 1, -1, ext, (nx[bi], ny[bj - 1], mz), ng))
        if bj == len(ny) - 1:
            faces.append(bc_face(q, BC_SYMMETRY, 1, 1, ext, ng))
        else:
            t = ids[(bi, bj + 1)]
            ifaces.append(iface_aligned(q, t, 1, 1, ext, (nx[bi], ny[bj + 1], mz), ng))
        faces += [bc_face(q, BC_SYMMETRY, 2, -1, ext, ng), bc_face(q, BC_SYMMETRY, 2, 1, ext, ng)]
    c = Case("multiblock_air_%dx%d_blocks" % (len(nx), len(ny)), s, None, blocks, faces, 100)
    c.interfaces = ifaces
    return c


def _partition(total, k, lo, hi, rng, fixed=()):
    """k block sizes in points, each in [lo, hi], whose shared-plane union
    spans `total` points (sum - (k - 1) == total); fixed: {index: size}."""
    fixed = dict(fixed)
    for _ in range(10000):
        sizes = [fixed.get(i, int(rng.integers(lo, hi + 1))) for i in range(k)]
        free = [i for i in range(k) if i not in fixed]
        short = total + k - 1 - sum(sizes)
        for i in free:  # spread the difference over the free sizes
            step = max(lo - sizes[i], min(hi - sizes[i], short))
            sizes[i] += step
            short -= step
        if short == 0:
            return sizes
    raise ValueError("no partition of %d points into %d sizes in [%d, %d]" % (total, k, lo, hi))


def block_layout(seed=37, n_layers=4, n_cols=3, rows=(3, 3, 3), extra_row=(1, 0), dims=(306, 200, 165),
                 ranges=((16, 192), (16, 96), (16, 64)), anchors=True):
    """Seeded uneven block layout of a box of dims points (shared planes):
    n_layers layers in k, each split in i into n_cols columns (its own
    split), each column split in j into rows[c] blocks (one more in the
    column extra_row = (layer, column)). Block sizes lie in `ranges`; with
    anchors, layer 0 holds a 16^3 block and layer 1 a 192 x 96 x 64 block.
    Returns a list of ((i0, j0, k0), (mx, my, mz)) in global point indices."""
    rng = np.random.default_rng(seed)
    NX, NY, NZ = dims
    (xlo, xhi), (ylo, yhi), (zlo, zhi) = ranges
    zs = _partition(NZ, n_layers, zlo, zhi, rng, {0: 16, 1: 64} if anchors else {})
    out = []
    k0 = 0
    for L in range(n_layers):
        fx = ({0: 16} if L == 0 else ({1: 192} if L == 1 else {})) if anchors else {}
        xs = _partition(NX, n_cols, xlo, xhi, rng, fx)
        i0 = 0
        for c in range(n_cols):
            nr = rows[c] + (1 if (L, c) == tuple(extra_row) else 0)
            fy = ({0: 16} if (L, c) == (0, 0) else ({0: 96} if (L, c) == (1, 1) else {})) if anchors else {}
            ys = _partition(NY, nr, ylo, yhi, rng, fy)
            j0 = 0
            for r in range(nr):
                out.append(((i0, j0, k0), (xs[c], ys[r], zs[L])))
                j0 += ys[r] - 1
            i0 += xs[c] - 1
        k0 += zs[L] - 1
    return out


def planar_layout(nx=(20, 17, 13), ny=(15, 19)):
    """A 2-D block layout for case_uneven_blocks: columns of nx[c] points and
    rows of ny[r] points sharing their face planes, every block one point
    deep in k (mz = 1). Returns [((i0, j0, 0), (mx, my, 1)), ...]."""
    out = []
    i0 = 0
    for mx in nx:
        j0 = 0
        for my in ny:
            out.append(((i0, j0, 0), (mx, my, 1)))
            j0 += my - 1
        i0 += mx - 1
    return out


def sst_freestream(state: dict, turbulence_intensity=0.01, viscosity_ratio=10.0) -> dict:
    """k, omega and mut of a free stream from its turbulence intensity and
    turbulent-to-laminar viscosity ratio (BoundCond.cpp:84-93): mut = ratio
    mu(T), k = 1.5 (U Tu)^2, omega = rho k / mut; air, Sutherland mu."""
    T = state["temperature"]
    mu = 1.716e-5 * (T / 273) ** 1.5 * (273 + 111) / (T + 111)
    mut = viscosity_ratio * mu
    k = 1.5 * state["velocity"] ** 2 * turbulence_intensity ** 2
    omega = state["density"] * k / mut
    out = dict(state)
    out.update(sv=[k, omega], mut=mut)
    return out


def wall_distance_j0(yg_shape_xyz, xs, ys, zs, i0, j0, k0, mx, my, mz, ng):
    """Distance of every ghosted point of a block to the wall node (global
    j = 0) of its own (i, k) grid line: the SST wall distance input of cases
    whose walls are the j = 0 plane (the reference's wall-distance search is
    pre-processing, outside this path)."""
    X = xs[k0:k0 + mz + 2 * ng, j0:j0 + my + 2 * ng, i0:i0 + mx + 2 * ng]
    Y = ys[k0:k0 + mz + 2 * ng, j0:j0 + my + 2 * ng, i0:i0 + mx + 2 * ng]
    Zc = zs[k0:k0 + mz + 2 * ng, j0:j0 + my + 2 * ng, i0:i0 + mx + 2 * ng]
    jw = ng  # global j = 0 in the ghosted global arrays
    Xw = xs[k0:k0 + mz + 2 * ng, jw:jw + 1, i0:i0 + mx + 2 * ng]
    Yw = ys[k0:k0 + mz + 2 * ng, jw:jw + 1, i0:i0 + mx + 2 * ng]
    Zw = zs[k0:k0 + mz + 2 * ng, jw:jw + 1, i0:i0 + mx + 2 * ng]
    return np.sqrt((X - Xw) ** 2 + (Y - Yw) ** 2 + (Zc - Zw) ** 2)


def case_uneven_blocks(seed=37, dx=1e-4, reconstruction=2, inviscid_scheme=4, mach=3.0, reynolds=1e7, T=300.0,
                       layout=None, rans_model=0, compressibility_correction=0) -> Case:
    """Uneven multi-block air case: the seeded layout of block_layout (37
    blocks from 16^3 to 192 x 96 x 64 joined by 1-to-1 interfaces, partial
    faces where neighbouring splits differ) in a warped box. Mach 3 air at
    Re = 1e7 / m (density from Sutherland's viscosity at T), a smooth
    tanh(y / 20 dy) boundary-layer profile, supersonic inflow at i-min,
    outflow at i-max, isothermal walls at T on every j-min block face (the
    12 blocks of the bottom row), far field at j-max, symmetry in k. layout:
    another block_layout (parity-sized runs). HLLC + MUSCL by default (the
    variant the reference build runs), laminar viscous fluxes, or k-omega SST
    with rans_model=2 (free stream at 1 % turbulence intensity and viscosity
    ratio 10, wall distance from wall_distance_j0)."""
    s = Scheme(mix_model=MIX_AIR, inviscid_scheme=inviscid_scheme, reconstruction=reconstruction, viscous_order=2,
               cfl=0.5, rans_model=rans_model, compressibility_correction=compressibility_correction)
    nt = 2 if rans_model == 2 else 0
    ng = s.ngg
    if layout is None:
        layout = block_layout(seed)
    NX = max(o[0] + e[0] for o, e in layout)
    NY = max(o[1] + e[1] for o, e in layout)
    NZ = max(o[2] + e[2] for o, e in layout)
    planar = NZ == 1  # a 2-D problem: no k faces, interfaces over k = 0 only
    for (_, e) in layout:
        if min(e[:2] if planar else e) < 2 * ng + 2:
            raise ValueError("block too small for the stencil: %s" % (e,))
    xg, yg, zg = grid_coordinates(NX, NY, NZ, ng + 1, dx, periodic_k=False)
    a = math.sqrt(GAMMA_AIR * R_U / MW_AIR * T)
    U = mach * a
    mu = 1.716e-5 * (T / 273) ** 1.5 * (273 + 111) / (T + 111)
    rho = reynolds * mu / U
    p = rho * R_U / MW_AIR * T
    ff = farfield_state(mach, T, p)
    if nt:
        ff = sst_freestream(ff)
    Xs, Ys, Zs = xg[1:-1, 1:-1, 1:-1], yg[1:-1, 1:-1, 1:-1], zg[1:-1, 1:-1, 1:-1]
    prof = np.tanh(np.maximum(Ys, 0.0) / (20 * dx))
    gbv = np.stack([np.full_like(Ys, rho), U * prof, 0 * Ys, 0 * Ys, np.full_like(Ys, p), np.full_like(Ys, T)])
    blocks, faces, ifaces = [], [], []
    for q, (o, e) in enumerate(layout):
        mx, my, mz = e
        b = HostBlock.allocate(mx, my, mz, ng, 5 + nt, 0, n_turb=nt)
        i0, j0, k0 = o
        sl = (slice(k0, k0 + mz + 2 * ng + 2), slice(j0, j0 + my + 2 * ng + 2), slice(i0, i0 + mx + 2 * ng + 2))
        fill_metric(b, np.ascontiguousarray(xg[sl]), np.ascontiguousarray(yg[sl]), np.ascontiguousarray(zg[sl]))
        b.arrays["bv"][...] = gbv[:, k0:k0 + mz + 2 * ng, j0:j0 + my + 2 * ng, i0:i0 + mx + 2 * ng]
        if nt:
            b.arrays["sv"][0] = ff["sv"][0]
            b.arrays["sv"][1] = ff["sv"][1]
            b.arrays["wall_distance"][...] = wall_distance_j0(None, Xs, Ys, Zs, i0, j0, k0, mx, my, mz, ng)
        blocks.append(b)
    wall = dict(wall_isothermal=1, wall_temperature=T)
    glob_hi = (NX - 1, NY - 1, NZ - 1)
    for q, (o, e) in enumerate(layout):
        lo = o
        hi = tuple(o[d] + e[d] - 1 for d in range(3))
        for d in range(3):
            for direction in (-1, 1):
                plane = lo[d] if direction < 0 else hi[d]
                if plane == (0 if direction < 0 else glob_hi[d]):
                    if d == 0:
                        faces.append(bc_face(q, BC_INFLOW if direction < 0 else BC_OUTFLOW, 0, direction, e, ng,
                                             ff if direction < 0 else None))
                    elif d == 1:
                        faces.append(bc_face(q, BC_WALL, 1, -1, e, ng, wall) if direction < 0 else
                                     bc_face(q, BC_FARFIELD, 1, 1, e, ng, ff))
                    elif not planar:
                        faces.append(bc_face(q, BC_SYMMETRY, 2, direction, e, ng))
                    continue
                # interior face: one interface patch per neighbour sharing this plane
                for t, (ot, et) in enumerate(layout):
                    if t == q:
                        continue
                    tlo = ot
                    thi = tuple(ot[c] + et[c] - 1 for c in range(3))
                    if (thi[d] if direction < 0 else tlo[d]) != plane:
                        continue
                    ov = []
                    for c in range(3):
                        if c == d:
                            continue
                        s0, s1 = max(lo[c], tlo[c]), min(hi[c], thi[c])
                        ov.append((c, s0, s1))
                    if any(s1 - s0 + 1 < 2 and not (planar and c == 2) for c, s0, s1 in ov):
                        continue
                    f = IfaceC()
                    f.block, f.target, f.face, f.direction = q, t, d, direction
                    for c in range(3):
                        f.loop_dir[c] = 1
                        f.target_loop_dir[c] = 1
                        f.src_tar[c] = c
                    if direction > 0:
                        f.range_start[d], f.range_end[d] = e[d] - 1, e[d] - 1 + ng
                        f.target_start[d] = 0
                    else:
                        f.range_start[d], f.range_end[d] = -ng, 0
                        f.target_start[d] = et[d] - 1 - ng
                    f.n_point[d] = ng + 1
                    for c, s0, s1 in ov:
                        f.range_start[c], f.range_end[c] = s0 - lo[c], s1 - lo[c]
                        f.target_start[c] = s0 - tlo[c]
                        f.n_point[c] = s1 - s0 + 1
                    ifaces.append(f)
    c = Case("uneven_blocks_%d_air%s_%dcells" % (len(layout), "_sst" if nt else "",
                                                  sum(e[0] * e[1] * e[2] for _, e in layout)), s, None,
             blocks, faces, 500)
    c.interfaces = ifaces
    return c


def make_steady(case: Case, implicit_method: int = 0, chem_src_method: Optional[int] = None,
                dplur_inner_step: int = 3, cfl: Optional[float] = None) -> Case:
    """The same blocks, faces and initial state advanced by the steady path
    (steady_simulation, src/SteadySim.cuh:15-137): local time stepping,
    explicit (implicit_method 0, with EPI / DA chemistry by chemSrcMethod)
    or DPLUR (1). Blocks are re-allocated with the one-ghost dq of DPLUR."""
    import copy

    s = copy.deepcopy(case.scheme)
    s.steady, s.implicit_method, s.dplur_inner_step = 1, implicit_method, dplur_inner_step
    if chem_src_method is not None:
        s.chemSrcMethod = chem_src_method
    if cfl is not None:
        s.cfl = cfl
    blocks = []
    for b in case.blocks:
        nb = HostBlock.allocate(b.mx, b.my, b.mz, b.ngg, b.n_var, b.n_spec, full=True, dq_ngg=s.dq_ngg,
                                n_turb=b.n_turb)
        for n, v in b.arrays.items():
            if n != "dq":
                nb.arrays[n][...] = v
        blocks.append(nb)
    c = Case(case.name + "_steady%d" % implicit_method, s, case.mech, blocks, list(case.faces), case.steps)
    c.interfaces = list(getattr(case, "interfaces", []) or [])
    return c


# ---------------------------------------------------------------------------
# the reacting mixing layer (9-species H2-air)
# ---------------------------------------------------------------------------
def mixture_state(mech: Mechanism, Y, T, p, mach):
    """rho, sound speed and velocity of a mixture stream (cfd::Inflow, src/BoundCond.cpp:7-80)."""
    t = mech.tables
    mw_inv = float(np.sum(Y / t["mw"]))
    W = 1.0 / mw_inv
    cp_i = np.empty(len(Y))
    for i in range(len(Y)):
        c = t["low_temp_coeff"][i] if T < t["t_mid"][i] else t["high_temp_coeff"][i]
        cp_i[i] = (c[0] + c[1] * T + c[2] * T ** 2 + c[3] * T ** 3 + c[4] * T ** 4) * R_U / t["mw"][i]
    cp = float(np.sum(Y * cp_i))
    cv = float(np.sum(Y * (cp_i - R_U / t["mw"])))
    gamma = cp / cv
    a = math.sqrt(gamma * R_U / W * T)
    rho = p * W / (R_U * T)
    return rho, a, mach * a


def case_mixing_layer(mx=256, my=256, mz=256, dx=1e-4, seed=2024, steps=200, full_host=False, mech=None,
                      cfl=0.4, rans_model=0, wall=False, compressibility_correction=0, mix_model=None) -> Case:
    """The reacting mixing layer: upper stream (y > 0) air (O2/N2 mass
    0.233/0.767) at 1500 K, Mach 2; lower stream H2/N2 (mole 0.3/0.7) at
    300 K, Mach 1.2; p = 1 atm; profiles blended by 0.5(1 + tanh(y / 8dy));
    seeded 1 % white-noise velocity perturbation (numpy PCG64; mz == 1: a 2-D
    layer, w = 0 and no k faces). 9-species,
    19-reaction H2-air mechanism, MUSCL (minmod) + AUSM+, laminar viscous
    flux, point-implicit chemistry tag (explicit under RK3, quirk A8), RK3 at
    CFL 0.4. Uniform Cartesian grid dx = dy = dz. Extrapolation (outflow)
    faces in x and y, periodic in z. rans_model=2: k-omega SST (Driver<FR,
    SST>) with k = 1.5 (0.01 U)^2 and omega = rho k / (10 * 1.8e-5) from
    the local stream speed U and density, the wall distance to the j = 0
    plane; wall=True makes j = 0 an isothermal 300 K wall (the fuel side).
    mech: any mechanism holding O2, N2 and H2 (species up to OSTC_MAX_SPEC);
    mix_model defaults to finite-rate chemistry when the mechanism has
    reactions and to the non-reacting mixture (MIX_MIXTURE) when it has none."""
    import chemdata

    mech = mech or chemdata.h2_air_9sp()
    if mix_model is None:
        mix_model = MIX_FR if mech.n_reac > 0 else MIX_MIXTURE
    s = Scheme(mix_model=mix_model, inviscid_scheme=3, reconstruction=2, limiter=0, viscous_order=2, chemSrcMethod=1,
               cfl=cfl, rans_model=rans_model, compressibility_correction=compressibility_correction)
    ng = s.ngg
    ns = mech.n_spec
    nt = 2 if rans_model == 2 else 0
    b = HostBlock.allocate(mx, my, mz, ng, 5 + ns + nt, ns, full=full_host, n_turb=nt)
    x, y, z = grid_coordinates(mx, my, mz, ng + 1, dx, warp=0.0)
    fill_metric(b, x, y, z)
    names = mech.names
    Y_air = np.zeros(ns)
    Y_air[names.index("O2")], Y_air[names.index("N2")] = 0.233, 0.767
    W = mech.tables["mw"]
    X_f = np.zeros(ns)
    X_f[names.index("H2")], X_f[names.index("N2")] = 0.3, 0.7
    Y_fuel = X_f * W / np.sum(X_f * W)
    p0 = 101325.0
    _, _, U_air = mixture_state(mech, Y_air, 1500.0, p0, 2.0)
    _, _, U_fuel = mixture_state(mech, Y_fuel, 300.0, p0, 1.2)
    P = b.plane()
    jj = (np.arange(-ng, my + ng) - my // 2) * dx
    f = 0.5 * (1 + np.tanh(jj / (8 * dx)))[None, :, None]
    f = np.broadcast_to(f, P)
    T = f * 1500.0 + (1 - f) * 300.0
    sv = b.arrays["sv"]
    for l in range(ns):
        sv[l] = f * Y_air[l] + (1 - f) * Y_fuel[l]
    mw_inv = np.zeros(P)
    for l in range(ns):
        mw_inv += sv[l] / W[l]
    U = f * U_air + (1 - f) * U_fuel
    rng = np.random.default_rng(seed)
    bv = b.arrays["bv"]
    bv[0] = p0 / (R_U * mw_inv * T)
    bv[1] = U * (1 + 0.01 * rng.uniform(-1, 1, P))
    bv[2] = 0.01 * U * rng.uniform(-1, 1, P)
    bv[3] = 0.01 * U * rng.uniform(-1, 1, P) if mz > 1 else 0.0  # a 2-D layer (mz == 1) has no w
    bv[4] = p0
    bv[5] = T
    if nt:
        tke = 1.5 * (0.01 * U) ** 2
        sv[ns] = tke
        sv[ns + 1] = bv[0] * tke / (10 * 1.8e-5)
        xs, ys, zs = x[1:-1, 1:-1, 1:-1], y[1:-1, 1:-1, 1:-1], z[1:-1, 1:-1, 1:-1]
        b.arrays["wall_distance"][...] = wall_distance_j0(None, xs, ys, zs, 0, 0, 0, mx, my, mz, ng)
    ext = (mx, my, mz)
    faces = [bc_face(0, BC_OUTFLOW, 0, -1, ext, ng), bc_face(0, BC_OUTFLOW, 0, 1, ext, ng),
             bc_face(0, BC_WALL, 1, -1, ext, ng, dict(wall_isothermal=1, wall_temperature=300.0)) if wall else
             bc_face(0, BC_OUTFLOW, 1, -1, ext, ng), bc_face(0, BC_OUTFLOW, 1, 1, ext, ng)]
    if mz > 1:
        faces += [bc_face(0, BC_PERIODIC, 2, -1, ext, ng), bc_face(0, BC_PERIODIC, 2, 1, ext, ng)]
    return Case("mixing_layer_h2air%s_%dx%dx%d" % ("_sst" if nt else "", mx, my, mz), s, mech, [b], faces, steps)


def case_premixed_box(mx=16, my=14, mz=8, dx=2e-3, T0=1400.0, seed=7, mech=None, chem_src_method=1,
                      cfl=0.4) -> Case:
    """A stoichiometric H2-air box (H2/O2/N2 mole 2/1/3.76) at T0 and 1 atm
    with +-5 % temperature and 10 m/s velocity noise (numpy PCG64, seeded).
    At dx = 2 mm the local time step (about 3e-7 s) makes the point-implicit
    chemistry treatments (EPI, DA) differ visibly from the explicit one while
    all of them stay bounded; at dx = 1 cm the chemistry is stiff enough that
    the explicit steady update diverges. MUSCL + AUSM+, laminar, extrapolation
    on every face."""
    import chemdata

    mech = mech or chemdata.h2_air_9sp()
    s = Scheme(mix_model=MIX_FR, inviscid_scheme=3, reconstruction=2, limiter=0, viscous_order=2,
               chemSrcMethod=chem_src_method, cfl=cfl)
    ng = s.ngg
    ns = mech.n_spec
    b = HostBlock.allocate(mx, my, mz, ng, 5 + ns, ns, full=True)
    x, y, z = grid_coordinates(mx, my, mz, ng + 1, dx, warp=0.0)
    fill_metric(b, x, y, z)
    names = mech.names
    W = mech.tables["mw"]
    X = np.zeros(ns)
    X[names.index("H2")], X[names.index("O2")], X[names.index("N2")] = 2.0, 1.0, 3.76
    Y = X * W / np.sum(X * W)
    P = b.plane()
    rng = np.random.default_rng(seed)
    T = T0 * (1 + 0.05 * rng.uniform(-1, 1, P))
    sv = b.arrays["sv"]
    for l in range(ns):
        sv[l] = Y[l]
    mw_inv = float(np.sum(Y / W))
    p0 = 101325.0
    bv = b.arrays["bv"]
    bv[0] = p0 / (R_U * mw_inv * T)
    bv[1] = 10.0 * rng.uniform(-1, 1, P)
    bv[2] = 10.0 * rng.uniform(-1, 1, P)
    bv[3] = 10.0 * rng.uniform(-1, 1, P)
    bv[4] = p0
    bv[5] = T
    ext = (mx, my, mz)
    faces = [bc_face(0, BC_OUTFLOW, d, e, ext, ng) for d in range(3) for e in (-1, 1)]
    return Case("premixed_h2air_%dx%dx%d" % (mx, my, mz), s, mech, [b], faces, 10)


# ---------------------------------------------------------------------------
# chemistry states for the point-implicit integrator and its surrogate
# ---------------------------------------------------------------------------
def species_elements(names):
    """element counts {element: array over species} parsed from species names
    like H2O2 (the elements of the H2-air mechanism: H, O, N)."""
    import re

    out = {}
    for k, nm in enumerate(names):
        for el, cnt in re.findall(r"([A-Z][a-z]?)(\d*)", nm):
            out.setdefault(el, np.zeros(len(names)))[k] += int(cnt or 1)
    return out


def sample_chem_states(mech: Mechanism, n: int, seed: int = 11, T_range=(300.0, 3000.0), p_atm=(0.5, 3.0),
                       dt_range=(1e-9, 1e-7)):
    """Seeded synthetic cell states with the value ranges of the mixing-layer
    runs: mixture fraction Z between the air stream (O2/N2 mass 0.233/0.767)
    and the fuel stream (H2/N2 mole 0.3/0.7), a progress variable c moving the
    unburnt mixture toward complete combustion products, radicals H, O, OH,
    HO2, H2O2 at log-uniform 1e-8..1e-3 (mass fractions renormalised), T
    uniform in T_range, p uniform in p_atm (atm), dt log-uniform in dt_range.
    Returns T[n], p[n], Y[n_spec][n], dt[n] as float64 numpy arrays."""
    rng = np.random.default_rng(seed)
    names, W = mech.names, mech.tables["mw"]
    ns = len(names)
    ix = {nm: names.index(nm) for nm in names}
    Y_air = np.zeros(ns)
    Y_air[ix["O2"]], Y_air[ix["N2"]] = 0.233, 0.767
    X_f = np.zeros(ns)
    X_f[ix["H2"]], X_f[ix["N2"]] = 0.3, 0.7
    Y_fuel = X_f * W / np.sum(X_f * W)
    Z = rng.uniform(0, 1, n)
    c = rng.uniform(0, 1, n)
    Yu = np.outer(Y_air, 1 - Z) + np.outer(Y_fuel, Z)  # [ns][n]
    # complete combustion 2 H2 + O2 -> 2 H2O of the limiting reactant
    nH2 = Yu[ix["H2"]] / W[ix["H2"]]
    nO2 = Yu[ix["O2"]] / W[ix["O2"]]
    burn = np.minimum(nH2, 2 * nO2) * c  # mol of H2 consumed per kg
    Y = Yu.copy()
    Y[ix["H2"]] -= burn * W[ix["H2"]]
    Y[ix["O2"]] -= 0.5 * burn * W[ix["O2"]]
    Y[ix["H2O"]] += burn * W[ix["H2O"]]
    for r in ("H", "O", "OH", "HO2", "H2O2"):
        Y[ix[r]] += 10 ** rng.uniform(-8, -3, n)
    Y = np.maximum(Y, 0)
    Y /= Y.sum(axis=0, keepdims=True)
    T = rng.uniform(T_range[0], T_range[1], n)
    p = 101325.0 * rng.uniform(p_atm[0], p_atm[1], n)
    dt = 10 ** rng.uniform(np.log10(dt_range[0]), np.log10(dt_range[1]), n)
    return T, p, np.ascontiguousarray(Y), dt


# ---------------------------------------------------------------------------
# the chemistry surrogate's network (csrc/mlp.cu)
# ---------------------------------------------------------------------------
SURR_IN, SURR_OUT, SURR_PARAMS = 12, 10, 137482


class Surrogate:
    """The 12-256-256-256-10 SiLU network of the chemistry surrogate on the
    GPU (BF16 weights and activations, FP32 accumulation and masters)."""

    def __init__(self, max_batch: int = 65536, seed: int = 1):
        h = C.c_void_p()
        check(lib().ostc_surrogate_create(max_batch, seed, C.byref(h)), "ostc_surrogate_create")
        self.h = h
        self.max_batch = max_batch

    def close(self):
        if self.h:
            lib().ostc_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _s():
        import torch

        return torch.cuda.current_stream().cuda_stream

    def set_scaling(self, in_mean, in_std, out_mean, out_std, in_min, in_max, out_r0=None):
        if out_r0 is None:
            out_r0 = np.zeros(SURR_OUT)
        arrs = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (in_mean, in_std, out_mean, out_std, in_min, in_max, out_r0)]
        self._scaling = arrs
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        check(lib().ostc_surrogate_set_scaling(self.h, *ptrs), "ostc_surrogate_set_scaling")

    def set_checks(self, elem_counts, elem_mass, tol_elem=1e-4, tol_T=1.0):
        a = np.ascontiguousarray(elem_counts, dtype=np.float64)
        m = np.ascontiguousarray(elem_mass, dtype=np.float64)
        self._checks = (a, m)
        check(lib().ostc_surrogate_set_checks(self.h, a.shape[0], a.shape[1], a.ctypes.data_as(C.POINTER(C.c_double)),
                                              m.ctypes.data_as(C.POINTER(C.c_double)), tol_elem, tol_T),
              "ostc_surrogate_set_checks")

    def params(self) -> np.ndarray:
        out = np.zeros(SURR_PARAMS, dtype=np.float32)
        check(lib().ostc_surrogate_get_params(self.h, out.ctypes.data), "ostc_surrogate_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().ostc_surrogate_set_params(self.h, p.ctypes.data), "ostc_surrogate_set_params")

    def forward(self, xs):
        import torch

        ys = torch.empty((xs.shape[0], SURR_OUT), dtype=torch.float32, device=xs.device)
        check(lib().ostc_surrogate_forward(self.h, xs.data_ptr(), xs.shape[0], ys.data_ptr(), self._s()),
              "ostc_surrogate_forward")
        return ys

    def inject_timeout(self, on: bool):
        """diagnostic: make the tensor-core kernels' bounded waits run out
        (their calls then return OSTC_ERR_TIMEOUT)"""
        check(lib().ostc_surrogate_inject_timeout(self.h, 1 if on else 0), "ostc_surrogate_inject_timeout")

    def forward_tc(self, xs):
        """the same network on the tcgen05 inference kernel"""
        import torch

        ys = torch.empty((xs.shape[0], SURR_OUT), dtype=torch.float32, device=xs.device)
        check(lib().ostc_surrogate_forward_tc(self.h, xs.data_ptr(), xs.shape[0], ys.data_ptr(), self._s()),
              "ostc_surrogate_forward_tc")
        return ys

    def gradients(self, xs, ys):
        g = np.zeros(SURR_PARAMS, dtype=np.float32)
        loss = C.c_float()
        check(lib().ostc_surrogate_gradients(self.h, xs.data_ptr(), ys.data_ptr(), xs.shape[0], g.ctypes.data,
                                             C.byref(loss), self._s()), "ostc_surrogate_gradients")
        return g, loss.value

    def train_step(self, xs, ys, lr, loss_dev=None):
        check(lib().ostc_surrogate_train_step(self.h, xs.data_ptr(), ys.data_ptr(), xs.shape[0], float(lr),
                                              loss_dev.data_ptr() if loss_dev is not None else None, self._s()),
              "ostc_surrogate_train_step")


# ---------------------------------------------------------------------------
# the reference's input files: grid, boundary and inner-face files, setup files
# ---------------------------------------------------------------------------
@dataclass
class Mesh:
    """A mesh read by ostc_mesh_read: per block the extents and the host
    arrays x, y, z, jac, metric (ngg ghost layers), the registered boundary
    faces (file labels, no state yet) and interfaces."""
    dimension: int
    ngg: int
    dims: List[tuple]
    coords: List[tuple]
    jac: List[np.ndarray]
    metric: List[np.ndarray]
    faces: List[BcFaceC]
    interfaces: List[IfaceC]


def read_mesh(grid_file, boundary_file, inner_file=None, ngg=2, grid_scale=1.0) -> Mesh:
    """cfd::Mesh's pre-processing (src/Mesh.cpp:550-588) through ostc_mesh_read"""
    h = C.c_void_p()
    check(lib().ostc_mesh_read(str(grid_file).encode(), str(boundary_file).encode(),
                               str(inner_file).encode() if inner_file else None, ngg, float(grid_scale), C.byref(h)),
          "ostc_mesh_read")
    try:
        nb, dim, nf, ni = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().ostc_mesh_sizes(h, C.byref(nb), C.byref(dim), C.byref(nf), C.byref(ni)), "ostc_mesh_sizes")
        dims, coords, jacs, mets = [], [], [], []
        for b in range(nb.value):
            mx, my, mz = C.c_int(), C.c_int(), C.c_int()
            check(lib().ostc_mesh_block(h, b, C.byref(mx), C.byref(my), C.byref(mz), None, None, None, None, None),
                  "ostc_mesh_block")
            shape = plane_shape(mx.value, my.value, mz.value, ngg)
            x, y, z, jac = (np.zeros(shape) for _ in range(4))
            met = np.zeros(shape, dtype=METRIC_DTYPE)
            check(lib().ostc_mesh_block(h, b, C.byref(mx), C.byref(my), C.byref(mz), x.ctypes.data, y.ctypes.data,
                                        z.ctypes.data, jac.ctypes.data, met.ctypes.data), "ostc_mesh_block")
            dims.append((mx.value, my.value, mz.value))
            coords.append((x, y, z))
            jacs.append(jac)
            mets.append(met)
        faces = (BcFaceC * max(1, nf.value))()
        ifaces = (IfaceC * max(1, ni.value))()
        check(lib().ostc_mesh_faces(h, faces), "ostc_mesh_faces")
        if ni.value:
            check(lib().ostc_mesh_interfaces(h, ifaces), "ostc_mesh_interfaces")
        return Mesh(dim.value, ngg, dims, coords, jacs, mets, list(faces)[:nf.value], list(ifaces)[:ni.value])
    finally:
        lib().ostc_mesh_destroy(h)


def read_setup(path) -> dict:
    """One of the reference's setup files, as Parameter::read_one_file parses
    it (src/Parameter.cpp:53-163): lines `type key = value` with type int,
    real, bool or string; `array <type> name { ... }` over one or more lines;
    `struct name { type key = value ... }`; // and ! start comments. Returns
    {key: value}, arrays as lists, structs as dicts."""
    conv = {"int": int, "real": float, "bool": lambda v: bool(int(v)), "string": str}
    out = {}
    lines = iter(Path(path).read_text().splitlines())
    for raw in lines:
        line = raw.split("//")[0].strip()
        if not line or raw.lstrip().startswith("!"):
            continue
        tok = line.split()
        if tok[0] in conv and len(tok) >= 4:
            out[tok[1]] = conv[tok[0]](tok[3])
        elif tok[0] == "array" and len(tok) >= 3:
            typ, name = tok[1], tok[2]
            body = line.split("{", 1)[1] if "{" in line else ""
            while "}" not in body:
                body += " " + next(lines).split("//")[0]
            body = body.split("}", 1)[0]
            out[name] = [conv[typ](v) for v in body.split()]
        elif tok[0] == "struct" and len(tok) >= 2:
            name, st = tok[1], {}
            for r in lines:
                r = r.split("//")[0].strip()
                if r.startswith("}"):
                    break
                t = r.split()
                if len(t) >= 4 and t[0] in conv:
                    st[t[1]] = conv[t[0]](t[3])
            out[name] = st
    return out


# default condition types of the labels no named condition claims (src/BoundCond.cu:228-252)
_LABEL_TYPES = {2: "wall", 3: "symmetry", 4: "farfield", 5: "inflow", 6: "outflow", 7: "subsonic_inflow",
                9: "back_pressure"}
_TYPE_LABELS = {"wall": BC_WALL, "symmetry": BC_SYMMETRY, "farfield": BC_FARFIELD, "inflow": BC_INFLOW,
                "outflow": BC_OUTFLOW, "subsonic_inflow": BC_SUBSONIC_INFLOW, "back_pressure": BC_BACK_PRESSURE}


def _nasa_cp(mech, l, T):
    """cp_k (J/kg/K) of the NASA-7 polynomials (src/Thermo.cu:47-61)"""
    t = mech.tables
    tt, c = T, t["high_temp_coeff"][l]
    if T < t["t_low"][l]:
        tt, c = t["t_low"][l], t["low_temp_coeff"][l]
    elif T < t["t_mid"][l]:
        c = t["low_temp_coeff"][l]
    return (c[0] + c[1] * tt + c[2] * tt ** 2 + c[3] * tt ** 3 + c[4] * tt ** 4) * R_U / t["mw"][l]


def inflow_state(info: dict, mech: Optional[Mechanism] = None) -> dict:
    """cfd::Inflow from its setup struct (src/BoundCond.cpp:7-90): (mach,
    pressure, temperature) or (density, velocity, pressure); u, v, w are the
    direction; species by name (mass fractions, or mole fractions when
    mole_or_mass = 0); the mixture's cp / cv ratio at the temperature"""
    ns = mech.n_spec if mech is not None else 0
    sv = np.zeros(ns)
    mw = MW_AIR
    if ns:
        for n, val in info.items():
            if n in mech.names:
                sv[mech.names.index(n)] = val
        W = mech.tables["mw"]
        if int(info.get("mole_or_mass", 1)) == 0:
            sv = sv * W / np.sum(sv * W)
        mw = 1.0 / np.sum(sv / W)
    T, p = info.get("temperature", -1.0), info.get("pressure", -1.0)
    rho = info.get("density", -1.0)
    if T < 0:
        T = p * mw / (rho * R_U)
    gamma = GAMMA_AIR
    if ns:
        cp = cv = 0.0
        for l in range(ns):
            c = _nasa_cp(mech, l, T)
            cp += sv[l] * c
            cv += sv[l] * (c - R_U / W[l])
        gamma = cp / cv
    c = math.sqrt(gamma * R_U / mw * T)
    mach = info.get("mach", -1.0)
    vel = info.get("velocity", 0.0)
    if mach < 0:
        mach = vel / c
    else:
        vel = mach * c
    if rho < 0:
        rho = p * mw / (R_U * T)
    return dict(density=rho, u=info.get("u", 1.0) * vel, v=info.get("v", 0.0) * vel, w=info.get("w", 0.0) * vel,
                pressure=p, temperature=T, velocity=vel, mut=0.0, sv=list(sv))


def boundary_setup(setup: dict, faces: List[BcFaceC], ngg: int, mech: Optional[Mechanism] = None) -> List[BcFaceC]:
    """DBoundCond::initialize_bc_on_GPU (src/BoundCond.cu:167-416) for faces
    read by read_mesh: each label takes the type of the named condition of
    `boundary_conditions` that claims it, else the default type of its number;
    inflow states from their structs (inflow_state), walls isothermal at the
    struct's temperature or adiabatic; wall faces trimmed by ngg on their
    tangential axes (src/BoundCond.cu:369-387). Returns new faces whose
    type_label is the condition type."""
    named = {}
    for name in setup.get("boundary_conditions", []):
        st = setup.get(name)
        if isinstance(st, dict) and "label" in st:
            named.setdefault(int(st["label"]), st)
    out = []
    for f in faces:
        st = named.get(f.type_label)
        typ = st.get("type") if st else _LABEL_TYPES.get(f.type_label)
        if typ not in _TYPE_LABELS:
            raise ValueError("boundary label %d: no condition type" % f.type_label)
        g = BcFaceC()
        C.pointer(g)[0] = f
        g.type_label = _TYPE_LABELS[typ]
        if typ == "inflow" and st:
            s = inflow_state(st, mech)
            for k in ("density", "u", "v", "w", "pressure", "temperature", "velocity", "mut"):
                setattr(g, k, float(s[k]))
            for l, y in enumerate(s["sv"]):
                g.sv[l] = float(y)
        if typ == "wall":
            if st and st.get("thermal_type", "isothermal") == "isothermal":
                g.wall_isothermal, g.wall_temperature = 1, float(st.get("temperature", 300.0))
            for a in range(3):
                if a != g.face:
                    g.range_start[a] += ngg
                    g.range_end[a] -= ngg
        out.append(g)
    return out


def write_reference_mesh(directory, dims, coords, boundaries, inner=None, n_file=0):
    """Writes a mesh in the reference's input-file formats under
    directory/input_files: grid/grid{n:>4}.grd (block count, extents, then x,
    y, z per block, i fastest), boundary_condition/boundary{n:>4}.txt (per
    block a count and rows i1 i2 j1 j2 k1 k2 label) and, with inner faces,
    boundary_condition/inner{n:>4}.txt (count line, faces per block, a title,
    then per face the source row with its 1-based block and the target row
    with the target's). coords: per block (x, y, z) arrays of the interior
    nodes, numpy layout [k][j][i]. Returns the three paths."""
    root = Path(directory) / "input_files"
    (root / "grid").mkdir(parents=True, exist_ok=True)
    (root / "boundary_condition").mkdir(parents=True, exist_ok=True)
    tag = "%4d" % n_file
    g = root / "grid" / ("grid%s.grd" % tag)
    with open(g, "w") as f:
        f.write("%12d\n" % len(dims))
        for d in dims:
            f.write("%12d%12d%12d\n" % tuple(d))
        for xyz in coords:
            for a in xyz:
                vals = np.asarray(a, dtype=np.float64).ravel()
                for q in range(0, vals.size, 3):
                    f.write("".join("%24.15f" % v for v in vals[q:q + 3]) + "\n")
    b = root / "boundary_condition" / ("boundary%s.txt" % tag)
    with open(b, "w") as f:
        for rows in boundaries:
            f.write("%12d\n" % len(rows))
            for r in rows:
                f.write("".join("%6d" % v for v in r) + "\n")
    i = None
    if inner is not None:
        i = root / "boundary_condition" / ("inner%s.txt" % tag)
        with open(i, "w") as f:
            f.write("%12d\n" % len(dims))
            f.write("".join("%12d" % len(rows) for rows in inner) + "\n")
            f.write(" imin  imax  jmin  jmax  kmin  kmax   id\n")
            for rows in inner:
                for src, tar in rows:
                    f.write("".join("%10d" % v for v in src) + "\n")
                    f.write("".join("%10d" % v for v in tar) + "\n")
    return g, b, i
