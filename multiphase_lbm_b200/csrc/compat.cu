// compat.cu -- the reference's three entry points (include/mlbm_compat.h)
// on top of the C ABI of include/mlbm.h.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/mlbm.h"
#include "../../include/mlbm_compat.h"

namespace {

int g_dims[3] = {400, 400, 400};
int g_storage = MLBM_STORE_F32;
mlbm_params g_params;
bool g_have_params = false;
mlbm_lattice* g_lat = nullptr;
float* g_rho = nullptr;       // the driver's rho array [x][y][z]
float* g_pressure = nullptr;  // the driver's pressure array

void die(mlbm_status st, const char* where) {
  std::fprintf(stderr, "libmlbm %s: %s: %s\n", where, mlbm_status_string(st),
               mlbm_last_error());
  std::exit(st);
}

void copy_back(const char* where) {
  if (g_rho)
    if (mlbm_status st = mlbm_download_field(g_lat, MLBM_FIELD_RHO,
                                             MLBM_DTYPE_F32, g_rho))
      die(st, where);
  if (g_pressure)
    if (mlbm_status st = mlbm_download_field(g_lat, MLBM_FIELD_PRESSURE,
                                             MLBM_DTYPE_F32, g_pressure))
      die(st, where);
}

}  // namespace

extern "C" {

void mlbm_compat_check(int e, const char* file, int line) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "CUDA Assert: %s %s %d\n",
                 cudaGetErrorString((cudaError_t)e), file, line);
    std::exit(e);
  }
}

void mlbm_compat_set_domain(int32_t lx, int32_t ly, int32_t lz) {
  g_dims[0] = lx;
  g_dims[1] = ly;
  g_dims[2] = lz;
}

void mlbm_compat_set_storage(int32_t storage) { g_storage = storage; }

// transfer_parameter, include/iteration_host.h:30-41
void transfer_parameter(float* tau, float* G, bool* carn_star, float* T_Tc,
                        float* rhol_spinodal, float* rhog_spinodal,
                        bool* inject_density, size_t* rho_inject_period,
                        float* rho_increment, float* rhos,
                        float* inject_position, size_t* statPeriod) {
  std::memset(&g_params, 0, sizeof g_params);
  g_params.tau = *tau;
  g_params.G = *G;
  g_params.carn_star = *carn_star;
  g_params.T_Tc = *T_Tc;
  g_params.rhol_spinodal = *rhol_spinodal;
  g_params.rhog_spinodal = *rhog_spinodal;
  g_params.inject_density = *inject_density;
  g_params.rho_inject_period = *rho_inject_period;
  g_params.rho_increment = *rho_increment;
  g_params.rhos = *rhos;
  g_params.inject_position = *inject_position;
  g_params.stat_period = *statPeriod;
  g_params.rho_shift = 1.0f;
  g_have_params = true;
}

// multiphaselbm_initialization, include/iteration_host.h:43-49
void multiphaselbm_initialization(void* rho_dd, void* psi_dd,
                                  void* pressure_dd, void* is_fluid_dd,
                                  void* collision_f_dd, void* stream_f_dd,
                                  void* force_dd) {
  (void)psi_dd;
  (void)collision_f_dd;
  (void)stream_f_dd;
  (void)force_dd;
  if (!g_have_params) die(MLBM_ERR_STATE, "initialization before transfer_parameter");
  g_rho = *static_cast<float**>(rho_dd);
  g_pressure = pressure_dd ? *static_cast<float**>(pressure_dd) : nullptr;
  const bool* fluid = *static_cast<bool**>(is_fluid_dd);
  mlbm_compat_release();
  int dev = 0;
  cudaGetDevice(&dev);
  if (mlbm_status st = mlbm_lattice_create(g_dims[0], g_dims[1], g_dims[2],
                                           g_storage, dev, &g_lat))
    die(st, "initialization");
  const size_t n = (size_t)g_dims[0] * g_dims[1] * g_dims[2];
  std::vector<uint8_t> mask(n);
  // the driver's arrays may be managed memory: read them through a copy
  std::vector<char> tmp(n * sizeof(bool));
  cudaMemcpy(tmp.data(), fluid, n * sizeof(bool), cudaMemcpyDefault);
  for (size_t k = 0; k < n; ++k) mask[k] = reinterpret_cast<bool*>(tmp.data())[k] ? 1 : 0;
  std::vector<float> rho(n);
  cudaMemcpy(rho.data(), g_rho, n * sizeof(float), cudaMemcpyDefault);
  if (mlbm_status st = mlbm_set_params(g_lat, &g_params)) die(st, "initialization");
  if (mlbm_status st = mlbm_upload_fluid_mask(g_lat, mask.data())) die(st, "initialization");
  if (mlbm_status st = mlbm_upload_rho(g_lat, rho.data())) die(st, "initialization");
  if (mlbm_status st = mlbm_initialize(g_lat)) die(st, "initialization");
  copy_back("initialization");
}

// multiphaselbm_iteration, include/iteration_host.h:56-57
void multiphaselbm_iteration(long step, size_t statPeriod, int reverse,
                             unsigned int inject_type) {
  if (!g_lat) die(MLBM_ERR_STATE, "iteration before initialization");
  if (mlbm_status st = mlbm_iterate(g_lat, step, 1, reverse, inject_type, 0))
    die(st, "iteration");
  if (statPeriod && (size_t)step % statPeriod == 0) copy_back("iteration");
}

mlbm_lattice* mlbm_compat_lattice(void) { return g_lat; }

void mlbm_compat_release(void) {
  if (g_lat) mlbm_lattice_destroy(g_lat);
  g_lat = nullptr;
}

}  // extern "C"
