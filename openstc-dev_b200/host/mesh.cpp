// mesh.cpp — host-side grid preprocessing of the path.
//
// ostc_metric_from_grid restates cfd::Block::compute_jac_metric
// (src/Mesh.cpp:259-521): second-order central differences of the node
// coordinates, Jacobian as the determinant of d(x,y,z)/d(xi,eta,zeta), and
// the metric as the inverse-transpose rows divided by the Jacobian. The
// reference evaluates the same formula on the interior and on six ghost
// slabs; here every point of [-ngg, m+ngg) is evaluated in one loop. A
// non-positive Jacobian inside the block is an error (Mesh.cpp:282-288);
// in the ghost slabs it takes the neighbour's value towards the block as
// the reference does (Mesh.cpp:321-326 and the following slabs).
#include <cmath>
#include <algorithm>
#include <cstring>

#include "../../include/ostc.h"

namespace {
struct G {  // coordinates with ngg+1 ghost layers
  const double *p;
  int mx, my, mz, g;
  long d2, d1, dt;
  G(const double *ptr, int mx_, int my_, int mz_, int g_) : p(ptr), mx(mx_), my(my_), mz(mz_), g(g_) {
    d2 = mx + 2 * g;
    d1 = (long)(my + 2 * g) * d2;
    dt = (d1 + d2 + 1) * g;
  }
  double operator()(int i, int j, int k) const { return p[(long)k * d1 + (long)j * d2 + i + dt]; }
};
}  // namespace

extern "C" ostc_status ostc_metric_from_grid(int mx, int my, int mz, int ngg, const double *x, const double *y,
                                             const double *z, double *jac_out, void *metric_out) {
  // mz == 1: a 2-D block, whose k ghost nodes the caller places at z(i, j, 0) + k as the
  // reference's grid reader does (Mesh.cpp:840-854); the plane k = 0 is then its interior
  // (Mesh.cpp:264-268)
  if (mx < 3 || my < 3 || (mz < 3 && mz != 1) || ngg < 1 || !x || !y || !z || !jac_out || !metric_out)
    return OSTC_ERR_INVALID_ARG;
  const G X(x, mx, my, mz, ngg + 1), Y(y, mx, my, mz, ngg + 1), Z(z, mx, my, mz, ngg + 1);
  const long d2 = mx + 2 * ngg, d1 = (long)(my + 2 * ngg) * d2, dt = (d1 + d2 + 1) * ngg;
  unsigned char *mo = (unsigned char *)metric_out;
  auto at = [&](int i, int j, int k) { return (long)k * d1 + (long)j * d2 + i + dt; };
  auto eval = [&](int i, int j, int k, double &jac, double m[9]) {
    const double dxd1 = (X(i + 1, j, k) - X(i - 1, j, k)) * 0.5, dyd1 = (Y(i + 1, j, k) - Y(i - 1, j, k)) * 0.5,
                 dzd1 = (Z(i + 1, j, k) - Z(i - 1, j, k)) * 0.5;
    const double dxd2 = (X(i, j + 1, k) - X(i, j - 1, k)) * 0.5, dyd2 = (Y(i, j + 1, k) - Y(i, j - 1, k)) * 0.5,
                 dzd2 = (Z(i, j + 1, k) - Z(i, j - 1, k)) * 0.5;
    const double dxd3 = (X(i, j, k + 1) - X(i, j, k - 1)) * 0.5, dyd3 = (Y(i, j, k + 1) - Y(i, j, k - 1)) * 0.5,
                 dzd3 = (Z(i, j, k + 1) - Z(i, j, k - 1)) * 0.5;
    jac = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 - dxd2 * dyd1 * dzd3 -
          dxd3 * dyd2 * dzd1;
    m[0] = (dyd2 * dzd3 - dyd3 * dzd2) / jac;
    m[1] = (dxd3 * dzd2 - dxd2 * dzd3) / jac;
    m[2] = (dxd2 * dyd3 - dxd3 * dyd2) / jac;
    m[3] = (dyd3 * dzd1 - dyd1 * dzd3) / jac;
    m[4] = (dxd1 * dzd3 - dxd3 * dzd1) / jac;
    m[5] = (dxd3 * dyd1 - dxd1 * dyd3) / jac;
    m[6] = (dyd1 * dzd2 - dyd2 * dzd1) / jac;
    m[7] = (dxd2 * dzd1 - dxd1 * dzd2) / jac;
    m[8] = (dxd1 * dyd2 - dxd2 * dyd1) / jac;
  };
  auto put = [&](int i, int j, int k, double jac, const double m[9]) {
    const long q = at(i, j, k);
    jac_out[q] = jac;
    unsigned char *rec = mo + 80 * q;
    const int bias = 4;  // gxl::Matrix<real,3,3,1>::bias_ = 1*(3+1)
    std::memcpy(rec, &bias, sizeof(int));
    std::memset(rec + 4, 0, 4);
    std::memcpy(rec + 8, m, 9 * sizeof(double));
  };
  // interior first, then ghosts from the inside out so a fallback copy sees its neighbour
  for (int k = 0; k < mz; ++k)
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        double jac, m[9];
        eval(i, j, k, jac, m);
        if (!(jac > 0)) return OSTC_ERR_NONPHYSICAL;
        put(i, j, k, jac, m);
      }
  for (int layer = 1; layer <= ngg; ++layer) {
    for (int k = -layer; k < mz + layer; ++k)
      for (int j = -layer; j < my + layer; ++j)
        for (int i = -layer; i < mx + layer; ++i) {
          const int di = i < 0 ? -i : (i >= mx ? i - mx + 1 : 0);
          const int dj = j < 0 ? -j : (j >= my ? j - my + 1 : 0);
          const int dk = k < 0 ? -k : (k >= mz ? k - mz + 1 : 0);
          if (std::max(di, std::max(dj, dk)) != layer) continue;
          double jac, m[9];
          eval(i, j, k, jac, m);
          if (!(jac > 0)) {
            const int ii = i < 0 ? i + 1 : (i >= mx ? i - 1 : i);
            const int jj = j < 0 ? j + 1 : (j >= my ? j - 1 : j);
            const int kk = k < 0 ? k + 1 : (k >= mz ? k - 1 : k);
            const long q = at(ii, jj, kk);
            jac = jac_out[q];
            std::memcpy(m, mo + 80 * q + 8, 9 * sizeof(double));
          }
          put(i, j, k, jac, m);
        }
  }
  return OSTC_OK;
}
