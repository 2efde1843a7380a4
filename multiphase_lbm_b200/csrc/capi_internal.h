// capi_internal.h -- the lattice handle behind the C ABI (not exported).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "../../include/mlbm.h"
#include "errors.h"
#include "lattice.cuh"
#include "update_tma.cuh"

namespace mlbm {
// Fluid-only population layout (compact.cuh).  Built from the mask on first
// use; the dense buffers stay allocated, and the state moves between the two
// layouts on demand.
struct CompactState {
  bool built = false;      // tables match the current mask
  bool active = false;     // the compact buffer holds the current state
  long long nfluid = 0, cs = 0;
  void* cpop = nullptr;        // [Q][cs] populations (T)
  uint2* cinfo = nullptr;      // [cs] (neighbour word, packed x, y, z)
  uint2* wtab = nullptr;       // [rows * wpr + 1] (mask word, wbase)
  bool two_pass_ok = false;    // the compact kernels fit the lattice
  uint32_t* wbase = nullptr;   // [rows * wpr + 1]
  long long cap = 0;           // cs the buffers were allocated for
  std::vector<long long> plane_start;  // [lz + 1] first compact index of each plane
  std::vector<uint32_t> row_start;     // [lz * ly + 1] first compact index of each row
  // one-pass step (band.cuh): the second population buffer and the tiling
  void* cpop_alt = nullptr;            // [Q][cs] populations (T)
  int band_rows = 4, band_planes = 24;  // requested rows per band, planes per chunk
  // stage size (compact slots) of the shape last launched, and its key
  int band_slot = 0, band_slot_rows = -1, band_slot_nb = -1, band_slot_storage = -1;
};

// Bound of the step kernels' device waits, and the test switch that makes
// one wait run out.
constexpr unsigned long long kDefaultWaitNs = 1000000000ull;  // 1 s
}  // namespace mlbm

struct mlbm_lattice {
  int device = 0;
  int storage = MLBM_STORE_F32;
  mlbm::Geom g{};
  mlbm_params params{};
  mlbm::Phys phys{};
  cudaStream_t stream = nullptr;
  bool stream_owned_sync = true;

  void* pop = nullptr;          // 19 planes of g.plane elements (T)
  void* rho = nullptr;          // density, R per node
  void* psi = nullptr;          // pseudopotential, R per node
  float* rho_init = nullptr;    // uploaded initial density (internal layout)
  uint32_t* mask = nullptr;     // 1 bit per node, 1 = fluid
  uint32_t* nbw = nullptr;      // per-node neighbour word (kernels.cuh)
  float* vel = nullptr;         // [node][3], written on request
  void* staging = nullptr;      // reference-layout transfer buffer
  size_t staging_bytes = 0;
  double* stats_scratch = nullptr;
  size_t stats_scratch_bytes = 0;
  int stats_wave = 0;           // resident blocks of the statistics kernel

  // update pass: z-march tiles and the TMA descriptor of the psi tensor
  mlbm::ZMarch zm{};
  alignas(64) CUtensorMap psi_map;

  int* err = nullptr;                      // device error flag (wait timeout)
  int step_kernel = 0;                     // MLBM_KERNEL_*
  mlbm::CompactState compact{};            // fluid-only layout (compact.cuh)

  unsigned long long wait_ns = mlbm::kDefaultWaitNs;  // bounded waits
  bool stall_test = false;  // the next step launch makes a wait run out
  int phase = 0;  // 0: post-collision at opp slots of own node; 1: pushed
  bool slab = false;  // planes 0 and lz - 1 are halo planes (slab.cu)
  bool has_params = false, has_mask = false, has_rho = false;
  bool initialized = false;
  bool vel_valid = false;
};

namespace mlbm {
mlbm_status cuda_fail(cudaError_t e, const char* where);
size_t pop_elem_bytes(int storage);
size_t real_bytes(int storage);
Geom make_geom(int lx, int ly, int lz);
// (Re)build the update pass's tile shape and psi tensor map.
mlbm_status setup_update(mlbm_lattice* lat, int rows, int planes);
struct StepArgs;
// The fluid-only layout (compact.cu).
mlbm_status compact_enter(mlbm_lattice* lat);   // dense -> compact state
mlbm_status compact_leave(mlbm_lattice* lat);   // compact -> dense state
mlbm_status compact_sync_dense(mlbm_lattice* lat);  // dense copy, stay compact
void compact_invalidate(mlbm_lattice* lat);     // the mask changed
void compact_free(mlbm_lattice* lat);
template <typename T>
mlbm_status launch_compact_two_pass(mlbm_lattice* lat, const StepArgs& a,
                                    bool write_u, bool write_rho);
template <typename T>
mlbm_status launch_compact_pass(mlbm_lattice* lat, const StepArgs& a, int pass,
                                bool write_u, bool write_rho);
bool compact_two_pass_supported(int lx, int ly, int lz, int storage);
// One-pass step over the compact layout with two buffers (compact.cu,
// band.cuh); starts and ends in AA phase 1.
template <typename T>
mlbm_status launch_compact_band(mlbm_lattice* lat, const StepArgs& a,
                                bool write_u, bool write_rho);
bool compact_band_supported(const mlbm_lattice* lat);
// Whether the lattice's bands fit shared memory (tables built); where they
// do not, BAND steps run as compact two-pass steps.
bool compact_band_fits(mlbm_lattice* lat);
mlbm_status compact_set_band_shape(mlbm_lattice* lat, int rows, int planes);
}  // namespace mlbm
