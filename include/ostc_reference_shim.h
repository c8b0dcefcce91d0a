/* ostc_reference_shim.h — the binding a maintainer of OpenSTC-dev adds to the
 * reference's own tree: an ostc_zone view of a block's device arrays, taken
 * from the reference's cfd::DZone (src/Field.h:13-71) as Field::h_ptr holds
 * it (src/Field.cu:133-251). Header-only C++; include it after the
 * reference's Field.h. The view points at the reference's arrays (no copy):
 * ostc_create on such zones runs this library's kernels on the reference's
 * own fields.
 *
 * dq_ngg: 0 for the RK3 path; 1 when the block's dq, dq0, dqk and spectral
 * radii carry the DPLUR ghost layer (src/Field.cu:209-221). */
#ifndef OSTC_REFERENCE_SHIM_H
#define OSTC_REFERENCE_SHIM_H

#include "ostc.h"

namespace ostc_from_reference {

template <class DZone>
inline ostc_zone to_ostc(const DZone &h, int dq_ngg = 0) {
  ostc_zone z{};
  auto &H = const_cast<DZone &>(h);  // ggxl arrays hand out their device pointers through non-const data()
  z.mx = h.mx;
  z.my = h.my;
  z.mz = h.mz;
  z.ngg = h.ngg;
  z.dq_ngg = dq_ngg;
  z.jac = H.jac.data();
  z.metric = H.metric.data();  // 80-byte gxl::Matrix<real,3,3,1> records
  z.wall_distance = H.wall_distance.data();
  z.cv = H.cv.data();
  z.bv = H.bv.data();
  z.sv = H.sv.data();
  z.bv_last = H.bv_last.data();
  z.vel = H.vel.data();
  z.acoustic_speed = H.acoustic_speed.data();
  z.mach = H.mach.data();
  z.mul = H.mul.data();
  z.thermal_conductivity = H.thermal_conductivity.data();
  z.rho_D = H.rho_D.data();
  z.gamma = H.gamma.data();
  z.cp = H.cp.data();
  z.chem_src_jac = H.chem_src_jac.data();
  z.mut = H.mut.data();
  z.turb_therm_cond = H.turb_therm_cond.data();
  z.turb_src_jac = H.turb_src_jac.data();
  z.dq = H.dq.data();
  z.dq0 = H.dq0.data();
  z.dqk = H.dqk.data();
  z.inv_spectr_rad = reinterpret_cast<double *>(H.inv_spectr_rad.data());  // real[3] per point, interleaved
  z.visc_spectr_rad = H.visc_spectr_rad.data();
  z.dt_local = H.dt_local.data();
  z.entropy_fix_delta = H.entropy_fix_delta.data();
  z.qn = H.qn.data();
  return z;
}

}  // namespace ostc_from_reference

#endif /* OSTC_REFERENCE_SHIM_H */
