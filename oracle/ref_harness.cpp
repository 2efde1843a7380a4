/*
 * ref_harness.cpp -- test infrastructure only (the oracle), never shipped.
 *
 * Runs the reference's OWN kernels and device functions on the host:
 * include/iteration_kernel.cuh and include/iteration_device.cuh are included
 * unmodified (through oracle/ref_shim.h), and one "CUDA thread" is executed
 * per lattice node from OpenMP loops.  It provides host definitions of the
 * three boundary functions the reference declares at
 * include/iteration_host.h:30-60 (its CUDA definitions are
 * src/iteration_host.cu:16-81), so the reference host driver
 * (src/multiphase_lbm.cu, linked into the same library) runs end to end on
 * the CPU, and a small extern "C" surface for the Python tests.
 *
 * Deviation from the reference GPU build (documented, deliberate):
 *   do_collision (include/iteration_kernel.cuh:32-41) runs compute_density
 *   and compute_force in the same launch, so neighbour psi values are a racy
 *   mix of two time levels on the GPU.  Here the collision is split into two
 *   sweeps over the lattice -- every fluid node's compute_density first, then
 *   every fluid node's compute_force + compute_velocity -- which is the
 *   race-free order the B200 implementation follows.
 *
 * The drainage boundary (inlet slab and outlet plane held at fixed density)
 * does not exist in the reference; the harness applies the same definition
 * the B200 kernels use: a fluid node with x < inlet_width (x >= lx -
 * outlet_width) has rho = rho_inlet (rho_outlet), psi = psi(rho), and its
 * post-collision populations are the rest equilibrium t_i * rho.
 */
#include "iteration_host.h"
#include "iteration_kernel.cuh"
#include "multiphase_lbm.h"

#include <cstdint>
#include <vector>

thread_local shim_dim3 blockIdx;
thread_local shim_dim3 threadIdx;
thread_local shim_dim3 blockDim;
thread_local shim_dim3 gridDim;

namespace {

int g_inlet_width = 0;
int g_outlet_width = 0;
real g_rho_inlet = 0.f;
real g_rho_outlet = 0.f;

inline void set_thread(size_t bx, size_t by, size_t bz, size_t gx) {
  blockIdx = {(unsigned)bx, (unsigned)by, (unsigned)bz};
  threadIdx = {0u, 0u, 0u};
  blockDim = {1u, 1u, 1u};
  gridDim = {(unsigned)gx, (unsigned)ly, (unsigned)lz};
}

inline int bc_kind(size_t x) {
  if ((int)x < g_inlet_width) return 1;
  if ((int)x >= (int)lx - g_outlet_width) return 2;
  return 0;
}

// Host storage for the fields when the harness owns them (ref_setup).
Realxyz* h_rho = nullptr;
Realxyz* h_psi = nullptr;
Realxyz* h_pressure = nullptr;
Boolxyz* h_fluid = nullptr;
RealxyzQ* h_fa = nullptr;
RealxyzQ* h_fb = nullptr;
Realxyz3* h_force = nullptr;

}  // namespace

// ---- host definitions of the reference boundary (include/iteration_host.h) --

void transfer_parameter(real* tau, real* G, bool* carn_star, real* T_Tc,
                        real* rhol_spinodal, real* rhog_spinodal,
                        bool* inject_density, size_t* rho_inject_period,
                        real* rho_increment, real* rhos, real* inject_position,
                        size_t* statPeriod) {
  dtau = *tau;
  dG = *G;
  dcarn_star = *carn_star;
  dT_Tc = *T_Tc;
  drhol_spinodal = *rhol_spinodal;
  drhog_spinodal = *rhog_spinodal;
  dinject_density = *inject_density;
  drho_inject_period = *rho_inject_period;
  drho_increment = *rho_increment;
  drhos = *rhos;
  dinject_position = *inject_position;
  dstatPeriod = *statPeriod;
}

void multiphaselbm_initialization(Realxyz** rho_dd, Realxyz** psi_dd,
                                  Realxyz** pressure_dd, Boolxyz** is_fluid_dd,
                                  RealxyzQ** collision_f_dd,
                                  RealxyzQ** stream_f_dd, Realxyz3** force_dd) {
  rho_d = *rho_dd;
  psi_d = *psi_dd;
  pressure_d = *pressure_dd;
  is_fluid_d = *is_fluid_dd;
  collision_f_d = *collision_f_dd;
  stream_f_d = *stream_f_dd;
  force_d = *force_dd;
#pragma omp parallel for schedule(static)
  for (size_t x = 0; x < lx; ++x)
    for (size_t y = 0; y < ly; ++y)
      for (size_t z = 0; z < lz; ++z) {
        set_thread(x, y, z, lx);
        multiphaselbm_init();
      }
}

void multiphaselbm_iteration(long step, size_t statPeriod, int reverse,
                             unsigned int inject_type) {
  (void)statPeriod;
  dinject_type = inject_type;
#pragma omp parallel for schedule(static)
  for (size_t xq = 0; xq < SCALE_LX * lx; ++xq)
    for (size_t y = 0; y < ly; ++y)
      for (size_t z = 0; z < lz; ++z) {
        set_thread(xq, y, z, SCALE_LX * lx);
        do_streaming();
      }
#pragma omp parallel for schedule(static)
  for (size_t x = 0; x < lx; ++x)
    for (size_t y = 0; y < ly; ++y)
      for (size_t z = 0; z < lz; ++z) {
        set_thread(x, y, z, lx);
        treat_boundary();
      }
  // do_collision, split into its two race-free sweeps.
#pragma omp parallel for schedule(static)
  for (size_t x = 0; x < lx; ++x)
    for (size_t y = 0; y < ly; ++y)
      for (size_t z = 0; z < lz; ++z) {
        if (!is_fluid_d[x][y][z]) continue;
        set_thread(x, y, z, lx);
        compute_density(step, x, y, z, reverse);
        int k = bc_kind(x);
        if (k) {
          real r = (k == 1) ? g_rho_inlet : g_rho_outlet;
          rho_d[x][y][z] = r;
          pressure_d[x][y][z] = dPress(r);
          psi_d[x][y][z] = dPsi(r);
        }
      }
#pragma omp parallel for schedule(static)
  for (size_t x = 0; x < lx; ++x)
    for (size_t y = 0; y < ly; ++y)
      for (size_t z = 0; z < lz; ++z) {
        if (!is_fluid_d[x][y][z]) continue;
        set_thread(x, y, z, lx);
        if (bc_kind(x)) {
          for (int i = 0; i < Q; ++i) stream_f_d[x][y][z][i] = t[i] * rho_d[x][y][z];
          force_d[x][y][z][0] = force_d[x][y][z][1] = force_d[x][y][z][2] = 0.f;
          continue;
        }
        compute_force(x, y, z);
        compute_velocity(x, y, z);
      }
  do_swap();
}

// ---- extern "C" surface for the tests ---------------------------------------

extern "C" {

struct ref_params {
  float tau, G, T_Tc, rhol_spinodal, rhog_spinodal, rho_increment, rhos,
      inject_position;
  int32_t carn_star, inject_density;
  uint64_t rho_inject_period, stat_period;
  int32_t inlet_width, outlet_width;
  float rho_inlet, rho_outlet;
};

int ref_lattice_dims(int32_t* dims) {
  dims[0] = lx;
  dims[1] = ly;
  dims[2] = lz;
  return 0;
}

void ref_free() {
  std::free(h_rho);
  std::free(h_psi);
  std::free(h_pressure);
  std::free(h_fluid);
  std::free(h_fa);
  std::free(h_fb);
  std::free(h_force);
  h_rho = h_psi = h_pressure = nullptr;
  h_fluid = nullptr;
  h_fa = h_fb = nullptr;
  h_force = nullptr;
}

// rho_xyz / fluid_xyz in the reference layout [x][y][z] (z fastest).
int ref_setup(const ref_params* p, const float* rho_xyz,
              const uint8_t* fluid_xyz) {
  ref_free();
  const size_t n = (size_t)lx * ly * lz;
  h_rho = (Realxyz*)std::calloc(n, sizeof(real));
  h_psi = (Realxyz*)std::calloc(n, sizeof(real));
  h_pressure = (Realxyz*)std::calloc(n, sizeof(real));
  h_fluid = (Boolxyz*)std::calloc(n, sizeof(bool));
  h_fa = (RealxyzQ*)std::calloc(n * Q, sizeof(real));
  h_fb = (RealxyzQ*)std::calloc(n * Q, sizeof(real));
  h_force = (Realxyz3*)std::calloc(n * 3, sizeof(real));
  if (!h_rho || !h_psi || !h_pressure || !h_fluid || !h_fa || !h_fb || !h_force)
    return 1;
  std::memcpy(h_rho, rho_xyz, n * sizeof(real));
  bool* fl = (bool*)h_fluid;
  for (size_t k = 0; k < n; ++k) fl[k] = fluid_xyz[k] != 0;

  real tau = p->tau, G = p->G, T_Tc = p->T_Tc, rl = p->rhol_spinodal,
       rg = p->rhog_spinodal, inc = p->rho_increment, rhos = p->rhos,
       ipos = p->inject_position;
  bool cs = p->carn_star != 0, inj = p->inject_density != 0;
  size_t per = p->rho_inject_period, sp = p->stat_period;
  g_inlet_width = p->inlet_width;
  g_outlet_width = p->outlet_width;
  g_rho_inlet = p->rho_inlet;
  g_rho_outlet = p->rho_outlet;
  transfer_parameter(&tau, &G, &cs, &T_Tc, &rl, &rg, &inj, &per, &inc, &rhos,
                     &ipos, &sp);
  multiphaselbm_initialization(&h_rho, &h_psi, &h_pressure, &h_fluid, &h_fa,
                               &h_fb, &h_force);
  return 0;
}

int ref_step(int64_t step0, int32_t nsteps, int32_t reverse,
             uint32_t inject_type) {
  for (int32_t s = 0; s < nsteps; ++s)
    multiphaselbm_iteration((long)(step0 + s), dstatPeriod, reverse,
                            inject_type);
  return 0;
}

// which: 0 rho, 1 pressure, 2 psi, 3 force [x][y][z][3],
//        4 post-collision populations collision_f [x][y][z][19]
int ref_get_field(int32_t which, float* out) {
  const size_t n = (size_t)lx * ly * lz;
  switch (which) {
    case 0: std::memcpy(out, rho_d, n * sizeof(real)); return 0;
    case 1: std::memcpy(out, pressure_d, n * sizeof(real)); return 0;
    case 2: std::memcpy(out, psi_d, n * sizeof(real)); return 0;
    case 3: std::memcpy(out, force_d, 3 * n * sizeof(real)); return 0;
    case 4: std::memcpy(out, collision_f_d, Q * n * sizeof(real)); return 0;
  }
  return 1;
}

// Runs the reference command-file parser and geometry builder
// (src/multiphase_lbm.cu:619-745) and copies out what it produced:
// rho [x][y][z], is_fluid [x][y][z], solid_number [x][y][z];
// info = {packing_density, solid_count, step, step_max, statPeriod, tau, G,
//         rhos, rho0, IniPerturbRate, rhol_spinodal, rhog_spinodal}.
int ref_driver_read(const char* cmdfile, float* rho_out, uint8_t* fluid_out,
                    int64_t* solid_number_out, double* info) {
  MultiphaseLBM* box = new MultiphaseLBM();
  box->read_data(cmdfile);
  const size_t n = (size_t)lx * ly * lz;
  std::memcpy(rho_out, box->drho, n * sizeof(real));
  const bool* fl = (const bool*)box->dis_fluid;
  const size_t* sn = (const size_t*)box->solid_number;
  for (size_t k = 0; k < n; ++k) {
    fluid_out[k] = fl[k] ? 1 : 0;
    solid_number_out[k] = (int64_t)sn[k];
  }
  info[0] = box->packing_density;
  info[1] = (double)box->solid_count;
  info[2] = (double)box->step;
  info[3] = (double)box->step_max;
  info[4] = (double)box->statPeriod;
  info[5] = box->tau;
  info[6] = box->G;
  info[7] = box->rhos;
  info[8] = box->rho0;
  info[9] = box->IniPerturbRate;
  info[10] = box->rhol_spinodal;
  info[11] = box->rhog_spinodal;
  std::free(box->dsolid_touch_liquid);  // the reference destructor leaks it
  delete box;
  return 0;
}

// Runs the reference statistics (calc_cluster, src/multiphase_lbm.cu:225-562,
// and the min/max part of write_stats, :1057-1072) on given fields.
// out = {saturation, avg_liq_p, avg_vap_p, avg_liq_rho, avg_vap_rho,
//        ratio_liquid_solid_boundary, ratio_liquid_vapor_boundary,
//        liq_cluster_count, gas_cluster_count, min_rho, max_rho, min_p, max_p}
int ref_driver_stats(const float* rho, const float* pressure,
                     const uint8_t* fluid, float rhol, float rhog,
                     double* out) {
  MultiphaseLBM* box = new MultiphaseLBM();
  box->rho0 = 1.f;
  box->IniPerturbRate = 0.f;
  box->resize_gpu();
  const size_t n = (size_t)lx * ly * lz;
  // resize_gpu never initialises the gas-cluster arrays (src/multiphase_lbm.cu
  // :146-156) and calc_cluster resets them at fluid nodes only, so the gas
  // flood would read uninitialised memory at solid nodes; start them at zero.
  std::memset(box->gas_cluster, 0, n * sizeof(bool));
  std::memset(box->gas_cluster_number, 0, n * sizeof(size_t));
  std::memcpy(box->drho, rho, n * sizeof(real));
  std::memcpy(box->dpressure, pressure, n * sizeof(real));
  bool* fl = (bool*)box->dis_fluid;
  for (size_t k = 0; k < n; ++k) fl[k] = fluid[k] != 0;
  box->rhol_spinodal = rhol;
  box->rhog_spinodal = rhog;
  box->vtkPeriod = 1u << 30;
  box->step = 1;
  box->calc_cluster();
  real mn = 1e9, mx = -1e-9, pmn = 1e9, pmx = -1e-9;
  for (size_t k = 0; k < n; ++k)
    if (fl[k]) {
      mn = std::min(rho[k], mn);
      mx = std::max(rho[k], mx);
      pmn = std::min(pressure[k], pmn);
      pmx = std::max(pressure[k], pmx);
    }
  out[0] = box->saturation_ratio;
  out[1] = box->average_liquid_pressure;
  out[2] = box->average_vapor_pressure;
  out[3] = box->average_liquid_density;
  out[4] = box->average_vapor_density;
  out[5] = box->ratio_liquid_solid_boundary;
  out[6] = box->ratio_liquid_vapor_boundary;
  out[7] = (double)box->liq_cluster_count;
  out[8] = (double)box->gas_cluster_count;
  out[9] = mn;
  out[10] = mx;
  out[11] = pmn;
  out[12] = pmx;
  std::free(box->dsolid_touch_liquid);  // the reference destructor leaks it
  delete box;
  return 0;
}

// calc_cluster with solid numbers (cluster order, wet coordination number,
// single-cluster radius): out = {liq_cluster_count, gas_cluster_count,
// cluster_order, wet_coord_num, max_r, ratio_liquid_solid_boundary,
// ratio_liquid_vapor_boundary, saturation}; liq/gas labels copied out.
int ref_driver_clusters(const float* rho, const float* pressure,
                        const uint8_t* fluid, const int64_t* solid_number,
                        int64_t solid_count, float rhol, float rhog,
                        double* out, int64_t* liq_labels, int64_t* gas_labels) {
  MultiphaseLBM* box = new MultiphaseLBM();
  box->rho0 = 1.f;
  box->IniPerturbRate = 0.f;
  box->resize_gpu();
  const size_t n = (size_t)lx * ly * lz;
  // resize_gpu never initialises the gas-cluster arrays (src/multiphase_lbm.cu
  // :146-156) and calc_cluster resets them at fluid nodes only, so the gas
  // flood would read uninitialised memory at solid nodes; start them at zero.
  std::memset(box->gas_cluster, 0, n * sizeof(bool));
  std::memset(box->gas_cluster_number, 0, n * sizeof(size_t));
  std::memcpy(box->drho, rho, n * sizeof(real));
  std::memcpy(box->dpressure, pressure, n * sizeof(real));
  bool* fl = (bool*)box->dis_fluid;
  size_t* sn = (size_t*)box->solid_number;
  for (size_t k = 0; k < n; ++k) {
    fl[k] = fluid[k] != 0;
    sn[k] = (size_t)solid_number[k];
  }
  box->solid_count = (size_t)solid_count;
  box->rhol_spinodal = rhol;
  box->rhog_spinodal = rhog;
  box->vtkPeriod = 1u << 30;
  box->step = 1;
  box->calc_cluster();
  out[0] = (double)box->liq_cluster_count;
  out[1] = (double)box->gas_cluster_count;
  out[2] = box->cluster_order;
  out[3] = box->wet_coord_num;
  out[4] = box->max_r;
  out[5] = box->ratio_liquid_solid_boundary;
  out[6] = box->ratio_liquid_vapor_boundary;
  out[7] = box->saturation_ratio;
  const size_t* ll = (const size_t*)box->liq_cluster_number;
  const size_t* gl = (const size_t*)box->gas_cluster_number;
  for (size_t k = 0; k < n; ++k) {
    liq_labels[k] = (int64_t)ll[k];
    gas_labels[k] = (int64_t)gl[k];
  }
  std::free(box->dsolid_touch_liquid);
  delete box;
  return 0;
}

}  // extern "C"
