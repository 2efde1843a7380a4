// output.cpp -- VTK output of the host driver: the legacy ASCII rectilinear
// grid of the reference's write_vtk_ascii (src/multiphase_lbm.cu:948-1054),
// same header, same fields (Zones, Density, Pressure, LiqClusters,
// GasClusters, Solids), same number formats and node order (x fastest).
#include <cstdio>
#include <string>
#include <vector>

#include "../../../include/mlbm.h"
#include "../../../include/mlbm_driver.h"
#include "../errors.h"

// The driver's result folder (driver.cpp).
std::string driver_result_folder(const mlbm_driver* d);
int driver_device(const mlbm_driver* d);

extern "C" mlbm_status mlbm_driver_write_vtk(mlbm_driver* d, int64_t num) {
  if (!d) return mlbm::set_error(MLBM_ERR_ARG, "null driver");
  mlbm_lattice* lat = mlbm_driver_lattice(d);
  if (!lat) return mlbm::set_error(MLBM_ERR_STATE, "write_vtk before run");
  int32_t dims[3];
  mlbm_driver_dims(d, dims);
  const int lx = dims[0], ly = dims[1], lz = dims[2];
  const size_t n = (size_t)lx * ly * lz;
  float* rho_in = nullptr;
  uint8_t* fluid = nullptr;
  int64_t* sn = nullptr;
  if (mlbm_status st = mlbm_driver_arrays(d, &rho_in, &fluid, &sn)) return st;
  std::vector<float> rho(n), pres(n);
  if (mlbm_status st = mlbm_download_field(lat, MLBM_FIELD_RHO, MLBM_DTYPE_F32, rho.data()))
    return st;
  if (mlbm_status st = mlbm_download_field(lat, MLBM_FIELD_PRESSURE, MLBM_DTYPE_F32, pres.data()))
    return st;
  mlbm_params p;
  mlbm_driver_params(d, &p);
  int64_t solid_count = 0;
  mlbm_driver_info(d, nullptr, nullptr, nullptr, nullptr, &solid_count, nullptr,
                   nullptr);
  std::vector<int64_t> liq(n), gas(n);
  mlbm_stats_row row{};
  if (mlbm_status st = mlbm_cluster_stats_gpu(
          rho.data(), fluid, sn, lx, ly, lz, p.rhol_spinodal, p.rhog_spinodal,
          solid_count, driver_device(d), liq.data(), gas.data(), &row))
    return st;

  char name[1024];
  std::snprintf(name, sizeof name, "%s/result%06lld.vtk",
                driver_result_folder(d).c_str(), (long long)num);
  FILE* f = std::fopen(name, "w");
  if (!f) return mlbm::set_error(MLBM_ERR_IO, "cannot create VTK file");
  const float step = 1.0f / lx;
  std::fprintf(f, "# vtk DataFile Version 2.0\n");
  std::fprintf(f, "Sortie domaine LB+LINK\n");
  std::fprintf(f, "ASCII\n");
  std::fprintf(f, "DATASET RECTILINEAR_GRID\n");
  std::fprintf(f, "DIMENSIONS %d %d %d\n", lx, ly, lz);
  std::fprintf(f, "X_COORDINATES %d float\n", lx);
  for (int i = 0; i < lx; ++i) std::fprintf(f, "%.4e ", (float)i * step);
  std::fprintf(f, "\n");
  std::fprintf(f, "Y_COORDINATES %d float\n", ly);
  for (int i = 0; i < ly; ++i) std::fprintf(f, "%.4e ", (float)i * step);
  std::fprintf(f, "\n");
  std::fprintf(f, "Z_COORDINATES %d float\n", lz);
  for (int i = 0; i < lz; ++i) std::fprintf(f, "%e ", (float)i * step);
  std::fprintf(f, "\n");
  std::fprintf(f, "POINT_DATA %zu\n", n);
  auto ridx = [&](int x, int y, int z) { return ((size_t)x * ly + y) * lz + z; };
  std::fprintf(f, "SCALARS Zones int 1\n");
  std::fprintf(f, "LOOKUP_TABLE default\n");
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x)
        std::fprintf(f, "%d\n", fluid[ridx(x, y, z)] ? 0 : 1);
  std::fprintf(f, "SCALARS Density float 1\n");
  std::fprintf(f, "LOOKUP_TABLE default\n");
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const size_t k = ridx(x, y, z);
        if (fluid[k]) std::fprintf(f, "%.4e\n", rho[k]);
        else std::fprintf(f, "0\n");
      }
  std::fprintf(f, "SCALARS Pressure float 1\n");
  std::fprintf(f, "LOOKUP_TABLE default\n");
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const size_t k = ridx(x, y, z);
        if (fluid[k]) std::fprintf(f, "%.4e\n", pres[k]);
        else std::fprintf(f, "0\n");
      }
  const char* names[3] = {"LiqClusters", "GasClusters", "Solids"};
  const int64_t* arrays[3] = {liq.data(), gas.data(), sn};
  for (int a = 0; a < 3; ++a) {
    std::fprintf(f, "SCALARS %s int 1\n", names[a]);
    std::fprintf(f, "LOOKUP_TABLE default\n");
    for (int z = 0; z < lz; ++z)
      for (int y = 0; y < ly; ++y)
        for (int x = 0; x < lx; ++x)
          std::fprintf(f, "%ld\n", (long)arrays[a][ridx(x, y, z)]);
  }
  std::fclose(f);
  return MLBM_OK;
}
