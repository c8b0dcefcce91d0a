// flowfield.h — host-side reader and writer of the reference's Tecplot
// binary flow-field file (flowfield.cpp); the C ABI entry points
// ostc_write_flowfield / ostc_read_flowfield (api.cu) move the device data.
#pragma once
#include <string>
#include <vector>

namespace ostc_io {

// one block's HOST planes, ghosted ColMajor with `ngg` layers (the layout of
// ostc_zone): the grid and the fields to write, the fields to read into
struct PltBlock {
  int mx = 0, my = 0, mz = 0, ngg = 0;
  const double *x = nullptr, *y = nullptr, *z = nullptr;
  const double *bv = nullptr, *mach = nullptr, *sv = nullptr, *mut = nullptr;
  double *bv_out = nullptr, *sv_out = nullptr;
};

// the file's variable names: x, y, z, density, u, v, w, pressure,
// temperature, mach, the species, and tke, omega, mut with SST
std::vector<std::string> variable_names(const std::vector<std::string> &species, bool sst);

// 0 on success; 1 the file could not be opened, 2 a write failed
int write_plt(const char *path, const std::vector<PltBlock> &blocks, const std::vector<std::string> &species,
              bool sst, int ngg_out, double solution_time);

// 0 on success; 1 the file could not be opened, 2 it is not in this layout,
// 3 a zone's extent does not fit its block. found: bit 0 species, bit 1 k and
// omega were in the file
int read_plt(const char *path, std::vector<PltBlock> &blocks, const std::vector<std::string> &species, bool sst,
             double *solution_time, int *found);

}  // namespace ostc_io
