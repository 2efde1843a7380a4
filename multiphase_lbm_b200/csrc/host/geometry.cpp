// geometry.cpp -- host geometry and initial density (include/mlbm_host.h).
//
// The voxeliser reproduces the reference's place_sphere
// (src/multiphase_lbm.cu:893-927) operation for operation -- float sample
// coordinates advanced by 1.0, float distance test, nearest() rounding in
// double (include/lbm_model.cuh:58) -- so solid masks are bit-identical.
// This file is compiled with -ffp-contract=off semantics in mind: no
// expression below may be contracted into an FMA (the build passes the flag).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "../../../include/mlbm_host.h"
#include "../errors.h"
#include "splitmix.h"

namespace {

inline long long ref_idx(int lx, int ly, int lz, int x, int y, int z) {
  (void)lx;
  return ((long long)x * ly + y) * lz + z;
}

// include/lbm_model.cuh:58
inline int nearest(float v) { return (int)std::floor(v + 0.5); }

inline int wrap_once(int v, int n) {
  // The reference wraps once (src/multiphase_lbm.cu:915-920); further wraps
  // keep spheres larger than the box in bounds.
  while (v < 0) v += n;
  while (v >= n) v -= n;
  return v;
}

using mlbm::SplitMix64;

bool blank(const std::string& s) {
  for (char c : s)
    if (!std::isspace((unsigned char)c)) return false;
  return true;
}

}  // namespace

extern "C" {

mlbm_status mlbm_place_sphere(uint8_t* is_fluid, int64_t* solid_number,
                              int32_t lx, int32_t ly, int32_t lz, float x,
                              float y, float z, float R, int64_t id) {
  if (!is_fluid || lx < 1 || ly < 1 || lz < 1)
    return mlbm::set_error(MLBM_ERR_ARG, "place_sphere: bad arguments");
  if (!(R >= 0.f) || !std::isfinite(x) || !std::isfinite(y) ||
      !std::isfinite(z) || !std::isfinite(R))
    return mlbm::set_error(MLBM_ERR_ARG, "place_sphere: non-finite sphere");
  const float xmin = x - R, ymin = y - R, zmin = z - R;
  const float xmax = x + R, ymax = y + R, zmax = z + R;
  const float R2 = R * R;
  for (float px = xmin; px <= xmax; px += 1.0f) {
    for (float py = ymin; py <= ymax; py += 1.0f) {
      for (float pz = zmin; pz <= zmax; pz += 1.0f) {
        const float dx = px - x;
        const float dy = py - y;
        const float dz = pz - z;
        const float dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
        const float dist2 = (dxx + dyy) + dzz;
        if (dist2 < R2) {
          const int nx = wrap_once(nearest(px), lx);
          const int ny = wrap_once(nearest(py), ly);
          const int nz = wrap_once(nearest(pz), lz);
          const long long k = ref_idx(lx, ly, lz, nx, ny, nz);
          is_fluid[k] = 0;
          if (solid_number) solid_number[k] = id;
        }
      }
    }
  }
  return MLBM_OK;
}

mlbm_status mlbm_read_positions(const char* path, float resolution,
                                uint8_t* is_fluid, int64_t* solid_number,
                                int32_t lx, int32_t ly, int32_t lz,
                                int64_t* count) {
  if (!path || !is_fluid || !count)
    return mlbm::set_error(MLBM_ERR_ARG, "read_positions: null argument");
  std::ifstream in(path);
  if (!in) {
    std::string m = std::string("cannot open positions file ") + path;
    return mlbm::set_error(MLBM_ERR_IO, m.c_str());
  }
  std::string line;
  int i = 0;
  float v[4] = {0, 0, 0, 0};
  long long lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (blank(line)) continue;
    errno = 0;
    char* end = nullptr;
    const double d = std::strtod(line.c_str(), &end);
    if (end == line.c_str() || errno == ERANGE) {
      char m[160];
      std::snprintf(m, sizeof m, "positions file %s: line %lld is not a number",
                    path, lineno);
      return mlbm::set_error(MLBM_ERR_PARSE, m);
    }
    // x = stod(line) * res, src/multiphase_lbm.cu:1112-1119
    v[i] = (float)(d * (double)resolution);
    if (++i == 4) {
      *count += 1;
      mlbm_status st = mlbm_place_sphere(is_fluid, solid_number, lx, ly, lz,
                                         v[0], v[1], v[2], v[3], *count);
      if (st) return st;
      i = 0;
    }
  }
  return MLBM_OK;
}

mlbm_status mlbm_init_density(float* rho, int32_t lx, int32_t ly, int32_t lz,
                              float rho0, float rate) {
  if (!rho || lx < 1 || ly < 1 || lz < 1)
    return mlbm::set_error(MLBM_ERR_ARG, "init_density: bad arguments");
  std::srand(1);
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const float u = (float)std::rand() / (float)RAND_MAX;
        rho[ref_idx(lx, ly, lz, x, y, z)] =
            (float)((double)rho0 * (1.0 + (double)rate * ((double)u - 0.5)));
      }
  return MLBM_OK;
}

mlbm_status mlbm_generate_packing(int32_t lx, int32_t ly, int32_t lz,
                                  float rmin, float rmax,
                                  double porosity_target, uint64_t seed,
                                  int64_t max_spheres, uint8_t* is_fluid,
                                  float* xyzr, int64_t* count,
                                  double* porosity) {
  if (!is_fluid || lx < 1 || ly < 1 || lz < 1 || !(rmin > 0.f) ||
      !(rmax >= rmin) || max_spheres < 0)
    return mlbm::set_error(MLBM_ERR_ARG, "generate_packing: bad arguments");
  const long long n = (long long)lx * ly * lz;
  std::memset(is_fluid, 1, (size_t)n);
  long long fluid = n;
  SplitMix64 rng{seed};
  int64_t placed = 0;
  // Count solids incrementally: voxelise into a scratch list of touched
  // nodes by diffing is_fluid before/after would be O(n); instead count
  // nodes flipped inside place_sphere's footprint.
  while ((double)fluid / (double)n > porosity_target && placed < max_spheres) {
    const float cx = rng.uniform() * (float)lx;
    const float cy = rng.uniform() * (float)ly;
    const float cz = rng.uniform() * (float)lz;
    const float r = rmin + rng.uniform() * (rmax - rmin);
    // footprint of the sphere (same loop bounds as place_sphere)
    long long flipped = 0;
    const float R2 = r * r;
    for (float px = cx - r; px <= cx + r; px += 1.0f)
      for (float py = cy - r; py <= cy + r; py += 1.0f)
        for (float pz = cz - r; pz <= cz + r; pz += 1.0f) {
          const float dx = px - cx, dy = py - cy, dz = pz - cz;
          const float dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
          if ((dxx + dyy) + dzz < R2) {
            const long long k =
                ref_idx(lx, ly, lz, wrap_once(nearest(px), lx),
                        wrap_once(nearest(py), ly), wrap_once(nearest(pz), lz));
            if (is_fluid[k]) {
              is_fluid[k] = 0;
              ++flipped;
            }
          }
        }
    fluid -= flipped;
    if (xyzr) {
      xyzr[4 * placed] = cx;
      xyzr[4 * placed + 1] = cy;
      xyzr[4 * placed + 2] = cz;
      xyzr[4 * placed + 3] = r;
    }
    ++placed;
  }
  if (count) *count = placed;
  if (porosity) *porosity = (double)fluid / (double)n;
  return MLBM_OK;
}

mlbm_status mlbm_generate_solids(uint8_t* is_fluid, int64_t* solid_number,
                                 int32_t lx, int32_t ly, int32_t lz,
                                 int32_t num, float rmin, float rmax,
                                 float xmin, float xmax, float ymin,
                                 float ymax, float zmin, float zmax,
                                 int64_t* count) {
  if (!is_fluid || !count)
    return mlbm::set_error(MLBM_ERR_ARG, "generate_solids: null argument");
  for (int i = 0; i < num; ++i) {
    // src/multiphase_lbm.cu:1096-1099 (float arithmetic on rand())
    const float r = (rmax - rmin) * ((float)std::rand() / (float)RAND_MAX) + rmin;
    const float x = (xmax - xmin) * ((float)std::rand() / (float)RAND_MAX) + xmin;
    const float y = (ymax - ymin) * ((float)std::rand() / (float)RAND_MAX) + ymin;
    const float z = (zmax - zmin) * ((float)std::rand() / (float)RAND_MAX) + zmin;
    *count += 1;
    mlbm_status st =
        mlbm_place_sphere(is_fluid, solid_number, lx, ly, lz, x, y, z, r, *count);
    if (st) return st;
  }
  return MLBM_OK;
}

mlbm_status mlbm_write_positions(const char* path, const float* xyzr,
                                 int64_t count) {
  if (!path || (!xyzr && count))
    return mlbm::set_error(MLBM_ERR_ARG, "write_positions: null argument");
  FILE* f = std::fopen(path, "w");
  if (!f) return mlbm::set_error(MLBM_ERR_IO, "cannot write positions file");
  for (int64_t k = 0; k < 4 * count; ++k) std::fprintf(f, "%.9g\n", xyzr[k]);
  std::fclose(f);
  return MLBM_OK;
}

double mlbm_packing_density(const uint8_t* is_fluid, int32_t lx, int32_t ly,
                            int32_t lz) {
  if (!is_fluid) return 0.0;
  const long long n = (long long)lx * ly * lz;
  long long solids = 0;
  for (long long k = 0; k < n; ++k) solids += is_fluid[k] ? 0 : 1;
  return n ? (double)solids / (double)n : 0.0;
}

mlbm_status mlbm_read_density_vtk(const char* path, float* rho, int32_t lx,
                                  int32_t ly, int32_t lz) {
  if (!path || !rho) return mlbm::set_error(MLBM_ERR_ARG, "null argument");
  std::ifstream in(path);
  if (!in) return mlbm::set_error(MLBM_ERR_IO, "cannot open density VTK file");
  std::string line;
  bool reading = false;
  long long k = 0;
  const long long n = (long long)lx * ly * lz;
  // src/multiphase_lbm.cu:118-131
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line == "SCALARS Pressure float 1") break;
    if (line == "SCALARS Density float 1") {
      reading = true;
      continue;
    }
    if (!reading || line == "LOOKUP_TABLE default") continue;
    if (k >= n) return mlbm::set_error(MLBM_ERR_PARSE, "too many density values");
    char* end = nullptr;
    const double d = std::strtod(line.c_str(), &end);
    if (end == line.c_str())
      return mlbm::set_error(MLBM_ERR_PARSE, "bad density value in VTK file");
    const int x = (int)(k % lx), y = (int)((k / lx) % ly), z = (int)(k / lx / ly);
    rho[ref_idx(lx, ly, lz, x, y, z)] = (float)d;
    ++k;
  }
  if (k != n) return mlbm::set_error(MLBM_ERR_PARSE, "VTK density block incomplete");
  return MLBM_OK;
}

}  // extern "C"
