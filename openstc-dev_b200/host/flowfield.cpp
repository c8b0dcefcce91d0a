// flowfield.cpp — the reference's restart / output file on the host: the
// Tecplot binary flow field that FieldIO::print_field writes
// (src/FieldIO.h:44-560) and read_flowfield reads back
// (src/Initialize.cuh:64-243, variable labels by identify_variable_labels,
// src/Initialize.cuh:246-310).
//
// Layout (V112, one ordered zone per block, every value nodal FP64):
//   header   "#!TDV112", int32 1, int32 file type 0, title "Solution file",
//            int32 n_var, the n_var names; per zone: float 299, name
//            "zone b", int32 -1 (parent), int32 -2 (strand), double solution
//            time, int32 -1 (color), 0 (ordered), 0 (nodal), 0, 0, int32
//            IMax, JMax, KMax, int32 0 (no auxiliary data); float 357
//   data     per zone: float 299, n_var int32 2 (double), int32 0 (no
//            passive), 0 (no sharing), -1 (no shared connectivity), the
//            min / max of every variable, then the variables one after the
//            other, i fastest, over [-ngg_out, m + ngg_out) per axis
//   strings  every character as an int32, then an int32 0
// Variables: x, y, z, density, u, v, w, pressure, temperature, mach, the
// species by name, tke and omega (SST), mut (SST).
//
// These are the host halves of ostc_write_flowfield / ostc_read_flowfield
// (api.cu), which move the device arrays.
#include "flowfield.h"

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>

namespace ostc_io {
namespace {

struct File {
  std::FILE *f = nullptr;
  explicit File(std::FILE *p) : f(p) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

bool put_i32(std::FILE *f, int32_t v) { return std::fwrite(&v, 4, 1, f) == 1; }
bool put_f32(std::FILE *f, float v) { return std::fwrite(&v, 4, 1, f) == 1; }
bool put_f64(std::FILE *f, double v) { return std::fwrite(&v, 8, 1, f) == 1; }
bool put_str(std::FILE *f, const std::string &s) {
  for (unsigned char c : s)
    if (!put_i32(f, (int32_t)c)) return false;
  return put_i32(f, 0);
}
bool get_i32(std::FILE *f, int32_t &v) { return std::fread(&v, 4, 1, f) == 1; }
bool get_f64(std::FILE *f, double &v) { return std::fread(&v, 8, 1, f) == 1; }
bool get_str(std::FILE *f, std::string &s) {
  s.clear();
  for (int n = 0; n < 4096; ++n) {
    int32_t c;
    if (!get_i32(f, c)) return false;
    if (c == 0) return true;
    s.push_back((char)c);
  }
  return false;  // no terminator within a sane length: not this format
}
bool skip(std::FILE *f, long long bytes) { return std::fseek(f, (long)bytes, SEEK_CUR) == 0; }

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// the values of plane `a` (ghosted ColMajor with g layers) over [-go, m+go)
template <typename F>
void for_range(const PltBlock &b, int go, F &&f) {
  const long long d2 = b.mx + 2 * b.ngg, d1 = (long long)(b.my + 2 * b.ngg) * d2;
  for (int k = -go; k < b.mz + go; ++k)
    for (int j = -go; j < b.my + go; ++j)
      for (int i = -go; i < b.mx + go; ++i) f((long long)(k + b.ngg) * d1 + (long long)(j + b.ngg) * d2 + i + b.ngg);
}

}  // namespace

std::vector<std::string> variable_names(const std::vector<std::string> &species, bool sst) {
  std::vector<std::string> v{"x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"};
  for (auto &s : species) v.push_back(s);
  if (sst) {
    v.push_back("tke");
    v.push_back("omega");
    v.push_back("mut");
  }
  return v;
}

int write_plt(const char *path, const std::vector<PltBlock> &blocks, const std::vector<std::string> &species,
              bool sst, int ngg_out, double solution_time) {
  File fh(std::fopen(path, "wb"));
  std::FILE *f = fh.f;
  if (!f) return 1;
  const auto names = variable_names(species, sst);
  const int n_var = (int)names.size();
  const int n_scalar = (int)species.size() + (sst ? 2 : 0);
  bool ok = std::fwrite("#!TDV112", 1, 8, f) == 8 && put_i32(f, 1) && put_i32(f, 0) && put_str(f, "Solution file") &&
            put_i32(f, n_var);
  for (auto &n : names) ok = ok && put_str(f, n);
  for (size_t b = 0; b < blocks.size() && ok; ++b) {
    const PltBlock &B = blocks[b];
    ok = put_f32(f, 299.0f) && put_str(f, "zone " + std::to_string(b)) && put_i32(f, -1) && put_i32(f, -2) &&
         put_f64(f, solution_time) && put_i32(f, -1) && put_i32(f, 0) && put_i32(f, 0) && put_i32(f, 0) &&
         put_i32(f, 0) && put_i32(f, B.mx + 2 * ngg_out) && put_i32(f, B.my + 2 * ngg_out) &&
         put_i32(f, B.mz + 2 * ngg_out) && put_i32(f, 0);
  }
  ok = ok && put_f32(f, 357.0f);
  for (size_t b = 0; b < blocks.size() && ok; ++b) {
    const PltBlock &B = blocks[b];
    const long long sz = (long long)(B.mx + 2 * B.ngg) * (B.my + 2 * B.ngg) * (B.mz + 2 * B.ngg);
    std::vector<const double *> planes{B.x, B.y, B.z};
    for (int l = 0; l < 6; ++l) planes.push_back(B.bv + l * sz);
    planes.push_back(B.mach);
    for (int l = 0; l < n_scalar; ++l) planes.push_back(B.sv + l * sz);
    if (sst) planes.push_back(B.mut);
    ok = put_f32(f, 299.0f);
    for (int l = 0; l < n_var && ok; ++l) ok = put_i32(f, 2);
    ok = ok && put_i32(f, 0) && put_i32(f, 0) && put_i32(f, -1);
    for (const double *p : planes) {
      double lo = p[0], hi = p[0];
      bool first = true;
      for_range(B, ngg_out, [&](long long q) {
        if (first) lo = hi = p[q], first = false;
        lo = std::min(lo, p[q]);
        hi = std::max(hi, p[q]);
      });
      ok = ok && put_f64(f, lo) && put_f64(f, hi);
    }
    std::vector<double> buf;
    buf.reserve((size_t)(B.mx + 2 * ngg_out) * (B.my + 2 * ngg_out) * (B.mz + 2 * ngg_out));
    for (const double *p : planes) {
      buf.clear();
      for_range(B, ngg_out, [&](long long q) { buf.push_back(p[q]); });
      ok = ok && std::fwrite(buf.data(), 8, buf.size(), f) == buf.size();
    }
  }
  return ok ? 0 : 2;
}

int read_plt(const char *path, std::vector<PltBlock> &blocks, const std::vector<std::string> &species, bool sst,
             double *solution_time, int *found) {
  File fh(std::fopen(path, "rb"));
  std::FILE *f = fh.f;
  if (!f) return 1;
  char magic[8];
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "#!TDV112", 8) != 0) return 2;
  std::string s;
  int32_t n_var = 0;
  if (!skip(f, 8) || !get_str(f, s) || !get_i32(f, n_var) || n_var < 3 || n_var > 4096) return 2;
  std::vector<std::string> names(n_var);
  for (auto &n : names)
    if (!get_str(f, n)) return 2;
  // labels as identify_variable_labels: 0-5 bv, 6.. species, then k, omega; -1 ignored
  const int ns = (int)species.size();
  int have = 0;
  std::vector<int> label(n_var, -1);
  for (int v = 0; v < n_var; ++v) {
    const std::string n = upper(names[v]);
    int l = -1;
    if (n == "DENSITY" || n == "ROE" || n == "RHO") l = 0;
    else if (n == "U") l = 1;
    else if (n == "V") l = 2;
    else if (n == "W") l = 3;
    else if (n == "P" || n == "PRESSURE") l = 4;
    else if (n == "T" || n == "TEMPERATURE") l = 5;
    else {
      for (int k = 0; k < ns; ++k)
        if (n == upper(species[k])) {
          l = 6 + k;
          have |= 1;
          break;
        }
      if (sst && (n == "K" || n == "TKE")) l = 6 + ns, have |= 2;
      if (sst && n == "OMEGA") l = 6 + ns + 1, have |= 2;
    }
    label[v] = v < 3 ? -1 : l;
  }
  const int nz = (int)blocks.size();
  std::vector<int32_t> ext(3 * (size_t)nz);
  double t = 0;
  for (int b = 0; b < nz; ++b) {
    if (!skip(f, 4) || !get_str(f, s) || !skip(f, 8) || !get_f64(f, t) || !skip(f, 20) || !get_i32(f, ext[3 * b]) ||
        !get_i32(f, ext[3 * b + 1]) || !get_i32(f, ext[3 * b + 2]) || !skip(f, 4))
      return 2;
  }
  if (!skip(f, 4)) return 2;
  for (int b = 0; b < nz; ++b) {
    PltBlock &B = blocks[b];
    const int fx = ext[3 * b], fy = ext[3 * b + 1], fz = ext[3 * b + 2];
    const int gf = (fx - B.mx) / 2;  // ghost layers in the file (the same on every axis)
    if (gf < 0 || gf > B.ngg || fx != B.mx + 2 * gf || fy != B.my + 2 * gf || fz != B.mz + 2 * gf) return 3;
    const long long N = (long long)fx * fy * fz;
    if (!skip(f, 4 + 4ll * n_var + 12 + 16ll * n_var) || !skip(f, 3 * N * 8)) return 2;
    const long long sz = (long long)(B.mx + 2 * B.ngg) * (B.my + 2 * B.ngg) * (B.mz + 2 * B.ngg);
    std::vector<double> buf((size_t)N);
    for (int v = 3; v < n_var; ++v) {
      double *dst = nullptr;
      const int l = label[v];
      if (l >= 0 && l < 6) dst = B.bv_out + l * sz;
      else if (l >= 6 && l < 6 + ns + (sst ? 2 : 0)) dst = B.sv_out + (l - 6) * sz;
      if (!dst) {
        if (!skip(f, N * 8)) return 2;
        continue;
      }
      if (std::fread(buf.data(), 8, (size_t)N, f) != (size_t)N) return 2;
      long long q = 0;
      for_range(B, gf, [&](long long g) { dst[g] = buf[q++]; });
    }
  }
  if (solution_time) *solution_time = t;
  if (found) *found = have;
  return 0;
}

}  // namespace ostc_io
