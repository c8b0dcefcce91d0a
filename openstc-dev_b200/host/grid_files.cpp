// grid_files.cpp — the grid pre-processing of the reference on the host: the
// text grid file, the boundary file and the inner-face file of
// input_files (cfd::Mesh::read_grid, read_boundary, read_inner_interface,
// src/Mesh.cpp:599-743), the registration of boundary faces and 1-to-1
// interfaces (Boundary / InnerFace::register_boundary, src/Mesh.cpp:14-178),
// the grid scale (src/Mesh.cpp:773-787), the ghost grid (init_ghost_grid and
// init_inner_ghost_grid, src/Mesh.cpp:789-987) and the metrics
// (ostc_metric_from_grid, the restatement of Block::compute_jac_metric).
// Single process: the parallel-interface file is not read.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ostc.h"

namespace {

int sgn(int v) { return (v > 0) - (v < 0); }

struct Coords {  // one coordinate with g ghost layers, (i, j, k) from -g
  int mx = 0, my = 0, mz = 0, g = 0;
  std::vector<double> v;
  void alloc(int x, int y, int z, int gg) {
    mx = x, my = y, mz = z, g = gg;
    v.assign((size_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g), 0.0);
  }
  double &operator()(int i, int j, int k) {
    return v[((size_t)(k + g) * (my + 2 * g) + (j + g)) * (mx + 2 * g) + (i + g)];
  }
};

struct Bnd {  // cfd::Boundary after register_boundary
  int rs[3], re[3], face = 0, direction = 1, label = 0;
};

struct Inner {  // cfd::InnerFace after register_boundary
  int rs[3], re[3], ts[3], te[3], target = 0, face = 0, direction = 1, tface = 0, tdirection = 1;
  int src_tar[3] = {0, 0, 0}, loop_dir[3], tloop_dir[3], n_point[3];
};

struct Blk {
  int mx, my, mz;
  Coords x, y, z;
  std::vector<Bnd> bnd;
  std::vector<Inner> inner;
  std::vector<double> jac;
  std::vector<unsigned char> met;
};

// Boundary::register_boundary (Mesh.cpp:14-32)
void register_boundary(Bnd &b, int ngg, int dim) {
  for (int i = 0; i < dim; ++i) {
    if (b.rs[i] == b.re[i]) {
      b.face = i;
      if (b.rs[i] == 0) b.direction = -1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (i == b.face) continue;
    if (b.re[i] < b.rs[i]) std::swap(b.re[i], b.rs[i]);
    b.rs[i] -= ngg;
    b.re[i] += ngg;
  }
  if (dim == 2) {
    b.rs[2] = -ngg;
    b.re[2] = ngg;
  }
}

// InnerFace::register_boundary (Mesh.cpp:44-178): 1-based ranges of the file
// (in 3-D a negative pair marks the tangential axis whose correspondence is
// set first) to the 0-based loop ranges over the ghost layers, the partner's
// start, the loop directions and the axis map src_tar
void register_inner(Inner &f, int ngg, int dim) {
  for (int i = 0; i < dim; ++i) {
    if (f.rs[i] == f.re[i]) {
      f.face = i;
      if (f.rs[i] == 1) f.direction = -1;
      f.rs[i] -= 1;
      f.re[i] -= 1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (f.ts[i] == f.te[i]) {
      f.tface = i;
      if (f.ts[i] == 1) f.tdirection = -1;
      f.ts[i] -= 1;
      f.te[i] -= 1;
      break;
    }
  }
  f.src_tar[f.tface] = -(f.direction * f.tdirection) * (f.face + 1);
  if (dim == 2) {
    const int nf = 1 - f.face, tnf = 1 - f.tface;
    f.rs[nf] = std::abs(f.rs[nf]) - 1;
    f.re[nf] = std::abs(f.re[nf]) - 1;
    f.ts[nf] = std::abs(f.ts[nf]) - 1;
    f.te[nf] = std::abs(f.te[nf]) - 1;
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
    f.src_tar[2] = 3;
    f.rs[2] = f.re[2] = f.ts[2] = f.te[2] = 0;
  } else {
    int nf = 0, tnf = 0;
    for (int i = 0; i < dim; ++i) {
      if (f.rs[i] < 0) {
        nf = i;
        f.rs[i] = -f.rs[i] - 1;
        f.re[i] = -f.re[i] - 1;
        break;
      }
    }
    for (int i = 0; i < dim; ++i) {
      if (f.ts[i] < 0) {
        tnf = i;
        f.ts[i] = -f.ts[i] - 1;
        f.te[i] = -f.te[i] - 1;
        break;
      }
    }
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
    nf = 3 - f.face - nf;
    tnf = 3 - f.tface - tnf;
    f.rs[nf] -= 1;
    f.re[nf] -= 1;
    f.ts[tnf] -= 1;
    f.te[tnf] -= 1;
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
  }
  // the face's loop covers its ghost layers and the coincident plane
  f.rs[f.face] = f.direction < 0 ? -ngg : f.re[f.face];
  f.re[f.face] = f.direction < 0 ? 0 : f.re[f.face] + ngg;
  const int st = sgn(f.src_tar[f.tface]);
  if (f.tdirection > 0)
    f.ts[f.tface] = st > 0 ? f.te[f.tface] - ngg : f.te[f.tface];
  else
    f.ts[f.tface] = st > 0 ? 0 : ngg;
  for (int i = 0; i < 3; ++i) {
    f.loop_dir[i] = f.rs[i] <= f.re[i] ? 1 : -1;
    f.tloop_dir[i] = sgn(f.src_tar[i]);
    f.src_tar[i] = std::abs(f.src_tar[i]) - 1;
    f.n_point[i] = std::abs(f.rs[i] - f.re[i]) + 1;
  }
}

bool in_coords(const Coords &C, int i, int j, int k) {
  return i >= -C.g && i < C.mx + C.g && j >= -C.g && j < C.my + C.g && k >= -C.g && k < C.mz + C.g;
}

// init_ghost_grid (Mesh.cpp:789-919): linear extrapolation along each axis
// (2-D: the k ghosts copy k = 0 shifted by k in z), the inner faces' ghosts
// from the partner block, then edges and corners by the parallelogram rule.
// false when an inner face reaches outside either block's ghosted grid
bool ghost_grid(std::vector<Blk> &blocks, int ngg, int dim) {
  for (auto &B : blocks) {
    const int mx = B.mx, my = B.my, mz = B.mz;
    Coords *c[3] = {&B.x, &B.y, &B.z};
    for (Coords *X : c) {
      for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) {
          for (int i = -1; i >= -ngg - 1; --i) (*X)(i, j, k) = 2 * (*X)(0, j, k) - (*X)(-i, j, k);
          for (int i = mx; i < mx + ngg + 1; ++i) (*X)(i, j, k) = 2 * (*X)(mx - 1, j, k) - (*X)(2 * (mx - 1) - i, j, k);
        }
      for (int k = 0; k < mz; ++k)
        for (int i = 0; i < mx; ++i) {
          for (int j = -1; j >= -ngg - 1; --j) (*X)(i, j, k) = 2 * (*X)(i, 0, k) - (*X)(i, -j, k);
          for (int j = my; j < my + ngg + 1; ++j) (*X)(i, j, k) = 2 * (*X)(i, my - 1, k) - (*X)(i, 2 * (my - 1) - j, k);
        }
    }
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        if (dim == 3) {
          for (Coords *X : c) {
            for (int k = -1; k >= -ngg - 1; --k) (*X)(i, j, k) = 2 * (*X)(i, j, 0) - (*X)(i, j, -k);
            for (int k = mz; k < mz + ngg + 1; ++k) (*X)(i, j, k) = 2 * (*X)(i, j, mz - 1) - (*X)(i, j, 2 * (mz - 1) - k);
          }
        } else {
          for (int k = -1; k >= -ngg - 1; --k) {
            B.x(i, j, k) = B.x(i, j, 0);
            B.y(i, j, k) = B.y(i, j, 0);
            B.z(i, j, k) = B.z(i, j, 0) + k;
          }
          for (int k = mz; k < mz + ngg + 1; ++k) {
            B.x(i, j, k) = B.x(i, j, mz - 1);
            B.y(i, j, k) = B.y(i, j, mz - 1);
            B.z(i, j, k) = B.z(i, j, mz - 1) + k - mz + 1;
          }
        }
      }
  }
  // init_inner_ghost_grid (Mesh.cpp:921-968): one layer beyond each inner
  // face's range, shifted away from the face, from the partner block
  for (auto &B : blocks) {
    for (const Inner &f : B.inner) {
      Blk &N = blocks[f.target];
      int mn[3] = {f.rs[0], f.rs[1], f.rs[2]}, mxr[3] = {f.re[0], f.re[1], f.re[2]};
      int mt[3] = {f.ts[0], f.ts[1], f.ts[2]};
      if (f.direction < 0) {
        mn[f.face] -= 1;
        mxr[f.face] -= 1;
      } else {
        mxr[f.face] += 1;
        mn[f.face] += 1;
      }
      mt[f.tface] += f.tdirection > 0 ? -1 : 1;
      int di[3];
      for (int i1 = mn[0]; f.loop_dir[0] * (i1 - mxr[0]) != 1; i1 += f.loop_dir[0]) {
        di[0] = i1 - mn[0];
        for (int j1 = mn[1]; f.loop_dir[1] * (j1 - mxr[1]) != 1; j1 += f.loop_dir[1]) {
          di[1] = j1 - mn[1];
          for (int k1 = mn[2]; f.loop_dir[2] * (k1 - mxr[2]) != 1; k1 += f.loop_dir[2]) {
            di[2] = k1 - mn[2];
            const int i2 = mt[0] + f.tloop_dir[0] * di[f.src_tar[0]];
            const int j2 = mt[1] + f.tloop_dir[1] * di[f.src_tar[1]];
            const int k2 = mt[2] + f.tloop_dir[2] * di[f.src_tar[2]];
            if (!in_coords(B.x, i1, j1, k1) || !in_coords(N.x, i2, j2, k2)) return false;
            B.x(i1, j1, k1) = N.x(i2, j2, k2);
            B.y(i1, j1, k1) = N.y(i2, j2, k2);
            B.z(i1, j1, k1) = N.z(i2, j2, k2);
          }
        }
      }
    }
  }
  // edges and corners (Mesh.cpp:866-918)
  for (auto &B : blocks) {
    const int mx = B.mx, my = B.my, mz = B.mz;
    for (Coords *X : {&B.x, &B.y, &B.z}) {
      Coords &P = *X;
      for (int i = 1; i <= ngg + 1; ++i)
        for (int j = 1; j <= ngg + 1; ++j)
          for (int k = 0; k < mz; ++k) {
            const int i1 = -i, j1 = -j, i2 = mx - 1 + i, j2 = my - 1 + j;
            P(i1, j1, k) = P(i1, 0, k) + P(0, j1, k) - P(0, 0, k);
            P(i2, j2, k) = P(i2, my - 1, k) + P(mx - 1, j2, k) - P(mx - 1, my - 1, k);
            P(i1, j2, k) = P(i1, my - 1, k) + P(0, j2, k) - P(0, my - 1, k);
            P(i2, j1, k) = P(i2, 0, k) + P(mx - 1, j1, k) - P(mx - 1, 0, k);
          }
      for (int i = 1; i <= ngg + 1; ++i)
        for (int j = 0; j < my; ++j)
          for (int k = 1; k <= ngg + 1; ++k) {
            const int i1 = -i, k1 = -k, i2 = mx - 1 + i, k2 = mz - 1 + k;
            P(i1, j, k1) = P(i1, j, 0) + P(0, j, k1) - P(0, j, 0);
            P(i2, j, k2) = P(i2, j, mz - 1) + P(mx - 1, j, k2) - P(mx - 1, j, mz - 1);
            P(i1, j, k2) = P(i1, j, mz - 1) + P(0, j, k2) - P(0, j, mz - 1);
            P(i2, j, k1) = P(i2, j, 0) + P(mx - 1, j, k1) - P(mx - 1, j, 0);
          }
      for (int i = -ngg - 1; i <= mx + ngg; ++i)
        for (int j = 1; j <= ngg + 1; ++j)
          for (int k = 1; k <= ngg + 1; ++k) {
            const int j1 = -j, k1 = -k, j2 = my - 1 + j, k2 = mz - 1 + k;
            P(i, j1, k1) = P(i, j1, 0) + P(i, 0, k1) - P(i, 0, 0);
            P(i, j2, k2) = P(i, j2, mz - 1) + P(i, my - 1, k2) - P(i, my - 1, mz - 1);
            P(i, j1, k2) = P(i, j1, mz - 1) + P(i, 0, k2) - P(i, 0, mz - 1);
            P(i, j2, k1) = P(i, j2, 0) + P(i, my - 1, k1) - P(i, my - 1, 0);
          }
    }
  }
  return true;
}

bool next_line(std::ifstream &f, std::string &s) { return (bool)std::getline(f, s); }

}  // namespace

struct ostc_mesh {
  int ngg = 0, dim = 3;
  std::vector<Blk> blocks;
};

extern "C" {

ostc_status ostc_mesh_read(const char *grid_file, const char *boundary_file, const char *inner_file, int ngg,
                           double grid_scale, ostc_mesh **out) {
  if (!grid_file || !boundary_file || !out || ngg < 1 || !(grid_scale > 0)) return OSTC_ERR_INVALID_ARG;
  *out = nullptr;
  auto m = new ostc_mesh();
  m->ngg = ngg;
  auto bad = [&](ostc_status s) {
    delete m;
    return s;
  };
  // read_grid (Mesh.cpp:599-652): block count, extents, then x, y, z of each block, i fastest
  std::ifstream grd(grid_file);
  if (!grd) return bad(OSTC_ERR_IO);
  std::string line;
  int nb = 0;
  if (!next_line(grd, line) || (nb = std::atoi(line.c_str())) < 1) return bad(OSTC_ERR_IO);
  m->blocks.resize(nb);
  for (auto &B : m->blocks) {
    if (!next_line(grd, line)) return bad(OSTC_ERR_IO);
    std::istringstream ls(line);
    if (!(ls >> B.mx >> B.my >> B.mz) || B.mx < 2 || B.my < 2 || B.mz < 1) return bad(OSTC_ERR_IO);
    for (Coords *X : {&B.x, &B.y, &B.z}) X->alloc(B.mx, B.my, B.mz, ngg + 1);
  }
  m->dim = m->blocks[0].mz == 1 ? 2 : 3;
  for (auto &B : m->blocks)
    for (Coords *X : {&B.x, &B.y, &B.z})
      for (int k = 0; k < B.mz; ++k)
        for (int j = 0; j < B.my; ++j)
          for (int i = 0; i < B.mx; ++i)
            if (!(grd >> (*X)(i, j, k))) return bad(OSTC_ERR_IO);
  // read_boundary (Mesh.cpp:654-676): per block a count, then i1 i2 j1 j2 k1 k2 label per face
  std::ifstream bnd(boundary_file);
  if (!bnd) return bad(OSTC_ERR_IO);
  for (auto &B : m->blocks) {
    if (!next_line(bnd, line)) return bad(OSTC_ERR_IO);
    const int n = std::atoi(line.c_str());
    for (int q = 0; q < n; ++q) {
      if (!next_line(bnd, line)) return bad(OSTC_ERR_IO);
      std::istringstream ls(line);
      Bnd b;
      if (!(ls >> b.rs[0] >> b.re[0] >> b.rs[1] >> b.re[1] >> b.rs[2] >> b.re[2] >> b.label)) return bad(OSTC_ERR_IO);
      register_boundary(b, ngg, m->dim);
      B.bnd.push_back(b);
    }
  }
  // read_inner_interface (Mesh.cpp:678-743): block count line, faces per block, a title line,
  // then per face the source range (and its block) and the target range and block, 1-based
  if (inner_file) {
    std::ifstream inn(inner_file);
    if (!inn) return bad(OSTC_ERR_IO);
    std::vector<int> n_face(nb);
    if (!next_line(inn, line)) return bad(OSTC_ERR_IO);
    for (int &n : n_face)
      if (!(inn >> n)) return bad(OSTC_ERR_IO);
    next_line(inn, line);
    next_line(inn, line);
    for (int b = 0; b < nb; ++b) {
      for (int q = 0; q < n_face[b]; ++q) {
        Inner f;
        int src_block = 0, tb = 0;
        if (!next_line(inn, line)) return bad(OSTC_ERR_IO);
        std::istringstream l1(line);
        if (!(l1 >> f.rs[0] >> f.re[0] >> f.rs[1] >> f.re[1] >> f.rs[2] >> f.re[2] >> src_block)) return bad(OSTC_ERR_IO);
        if (!next_line(inn, line)) return bad(OSTC_ERR_IO);
        std::istringstream l2(line);
        if (!(l2 >> f.ts[0] >> f.te[0] >> f.ts[1] >> f.te[1] >> f.ts[2] >> f.te[2] >> tb)) return bad(OSTC_ERR_IO);
        f.target = tb - 1;
        if (f.target < 0 || f.target >= nb) return bad(OSTC_ERR_IO);
        register_inner(f, ngg, m->dim);
        m->blocks[b].inner.push_back(f);
      }
    }
  }
  // scale (Mesh.cpp:773-787), then the ghost grid and the metrics
  if (std::abs(grid_scale - 1.0) > 1e-15)
    for (auto &B : m->blocks)
      for (Coords *X : {&B.x, &B.y, &B.z})
        for (auto &v : X->v) v *= grid_scale;
  if (!ghost_grid(m->blocks, ngg, m->dim)) return bad(OSTC_ERR_INVALID_ARG);
  for (auto &B : m->blocks) {
    const size_t np = (size_t)(B.mx + 2 * ngg) * (B.my + 2 * ngg) * (B.mz + 2 * ngg);
    B.jac.assign(np, 0.0);
    B.met.assign(np * 80, 0);
    const ostc_status st = ostc_metric_from_grid(B.mx, B.my, B.mz, ngg, B.x.v.data(), B.y.v.data(), B.z.v.data(),
                                                 B.jac.data(), B.met.data());
    if (st != OSTC_OK) return bad(st);
  }
  *out = m;
  return OSTC_OK;
}

ostc_status ostc_mesh_destroy(ostc_mesh *m) {
  delete m;
  return OSTC_OK;
}

ostc_status ostc_mesh_sizes(const ostc_mesh *m, int *n_blocks, int *dimension, int *n_faces, int *n_interfaces) {
  if (!m) return OSTC_ERR_INVALID_ARG;
  int nf = 0, ni = 0;
  for (auto &B : m->blocks) nf += (int)B.bnd.size(), ni += (int)B.inner.size();
  if (n_blocks) *n_blocks = (int)m->blocks.size();
  if (dimension) *dimension = m->dim;
  if (n_faces) *n_faces = nf;
  if (n_interfaces) *n_interfaces = ni;
  return OSTC_OK;
}

ostc_status ostc_mesh_block(const ostc_mesh *m, int b, int *mx, int *my, int *mz, double *x, double *y, double *z,
                            double *jac, void *metric) {
  if (!m || b < 0 || b >= (int)m->blocks.size()) return OSTC_ERR_INVALID_ARG;
  const Blk &B = m->blocks[b];
  if (mx) *mx = B.mx;
  if (my) *my = B.my;
  if (mz) *mz = B.mz;
  const int g = m->ngg;
  const long long d2 = B.mx + 2 * g, d1 = (long long)(B.my + 2 * g) * d2;
  const Coords *c[3] = {&B.x, &B.y, &B.z};
  double *o[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) {
    if (!o[a]) continue;
    Coords &C = const_cast<Coords &>(*c[a]);
    for (int k = -g; k < B.mz + g; ++k)
      for (int j = -g; j < B.my + g; ++j)
        for (int i = -g; i < B.mx + g; ++i) o[a][(k + g) * d1 + (j + g) * d2 + i + g] = C(i, j, k);
  }
  if (jac) std::copy(B.jac.begin(), B.jac.end(), jac);
  if (metric) std::copy(B.met.begin(), B.met.end(), (unsigned char *)metric);
  return OSTC_OK;
}

ostc_status ostc_mesh_faces(const ostc_mesh *m, ostc_bc_face *faces) {
  if (!m || !faces) return OSTC_ERR_INVALID_ARG;
  int q = 0;
  for (size_t b = 0; b < m->blocks.size(); ++b)
    for (const Bnd &s : m->blocks[b].bnd) {
      ostc_bc_face &f = faces[q++];
      std::memset(&f, 0, sizeof(f));
      f.block = (int)b;
      f.type_label = s.label;
      f.face = s.face;
      f.direction = s.direction;
      for (int a = 0; a < 3; ++a) f.range_start[a] = s.rs[a], f.range_end[a] = s.re[a];
    }
  return OSTC_OK;
}

ostc_status ostc_mesh_interfaces(const ostc_mesh *m, ostc_interface *faces) {
  if (!m || !faces) return OSTC_ERR_INVALID_ARG;
  int q = 0;
  for (size_t b = 0; b < m->blocks.size(); ++b)
    for (const Inner &s : m->blocks[b].inner) {
      ostc_interface &f = faces[q++];
      f.block = (int)b;
      f.target = s.target;
      f.face = s.face;
      f.direction = s.direction;
      for (int a = 0; a < 3; ++a) {
        f.range_start[a] = s.rs[a];
        f.range_end[a] = s.re[a];
        f.target_start[a] = s.ts[a];
        f.loop_dir[a] = s.loop_dir[a];
        f.target_loop_dir[a] = s.tloop_dir[a];
        f.src_tar[a] = s.src_tar[a];
        f.n_point[a] = s.n_point[a];
      }
    }
  return OSTC_OK;
}

}  // extern "C"
