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
// Launch geometry of the fused persistent time step (persistent.cuh).
struct FusedShape {
  int Tx, Ty, ntx, nty, ntiles, threads, L;
  size_t smem;
  bool ok;      // false: the fused kernel cannot run this lattice
  bool chosen;  // tile shape fixed (by tuning or at the first launch)
};

// Fluid-only population layout and tiling of the single-pass step
// (compact.cuh).  Built from the mask on first use; the dense buffers stay
// allocated, and the state moves between the two layouts on demand.
struct CompactState {
  bool supported = false;  // storage and lattice shape allow the step
  bool built = false;      // tables match the current mask
  bool active = false;     // the compact buffer holds the current state
  bool parts_valid = false;  // part sums match the state (single-pass step)
  long long nfluid = 0, cs = 0;
  void* cpop = nullptr;        // [Q][cs] populations (T)
  float* part = nullptr;       // [2][4][cs] part sums of rho (two sets)
  uint32_t* cnb = nullptr;     // [cs] neighbour words in compact order
  uint2* cinfo = nullptr;      // [cs] (neighbour word, packed x, y, z)
  uint2* wtab = nullptr;       // [rows * wpr + 1] (mask word, wbase)
  bool two_pass_ok = false;    // the compact two-pass kernels fit the lattice
  uint32_t* wbase = nullptr;   // [rows * wpr + 1]
  int* tabs = nullptr;         // ytab[ly], ztab[lz], ystart[nty+1], zstart[nzc+1]
  long long cap = 0;           // cs the buffers were allocated for
  int rows = 4, planes = 8;    // requested tile height and chunk depth
  int nty = 0, nzc = 0, rows_max = 0;
  size_t smem = 0;
  // wavefront step (wave.cuh)
  std::vector<long long> plane_start;  // [lz + 1] first compact index of each plane
  int4* wave_items = nullptr;          // work list
  unsigned* wave_need = nullptr;       // [lz] density tiles per plane
  unsigned* wave_ctl = nullptr;        // ticket[2], done[2][lz]
  int wave_nitems = 0;
  int wave_tile = 1024, wave_lookahead = 4;  // nodes per item, planes ahead
  int wave_par = 0;                    // counter set of the next launch
  int wave_grid[2] = {0, 0};           // persistent CTAs per AA phase
  bool wave_built = false;             // work list matches tables and shape
  // one-pass step (band.cuh): the second population buffer and the tiling
  void* cpop_alt = nullptr;            // [Q][cs] populations (T)
  int band_rows = 4, band_planes = 24;  // requested rows per band, planes per chunk
};
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

  // update pass: z-march tiles and the TMA descriptor of the psi tensor
  mlbm::ZMarch zm{};
  alignas(64) CUtensorMap psi_map;

  // fused persistent step
  mlbm::FusedShape fused{};
  unsigned long long fused_epoch = 0;      // progress-counter base
  unsigned* pdone = nullptr;               // per-tile progress counters
  int* err = nullptr;                      // device error flag (wait timeout)
  int step_kernel = 0;                     // MLBM_KERNEL_*
  mlbm::CompactState compact{};            // single-pass step (compact.cuh)

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
FusedShape fused_shape(const Geom& g, int storage, int ty_hint, int lag);
int max_tiles(const Geom& g);
// (Re)build the update pass's tile shape and psi tensor map.
mlbm_status setup_update(mlbm_lattice* lat, int rows, int planes);
struct StepArgs;
template <typename T>
mlbm_status launch_fused(mlbm_lattice* lat, const StepArgs& a, int out);
// Single-pass step over the compact layout (compact.cu).
bool compact_supported(int lx, int ly, int lz, int storage);
mlbm_status compact_set_shape(mlbm_lattice* lat, int rows, int planes);
mlbm_status compact_enter(mlbm_lattice* lat);   // dense -> compact state
mlbm_status compact_leave(mlbm_lattice* lat);   // compact -> dense state
mlbm_status compact_sync_dense(mlbm_lattice* lat);  // dense copy, stay compact
void compact_invalidate(mlbm_lattice* lat);     // the mask changed
void compact_free(mlbm_lattice* lat);
template <typename T>
mlbm_status launch_compact(mlbm_lattice* lat, const StepArgs& a, int out);
template <typename T>
mlbm_status launch_compact_two_pass(mlbm_lattice* lat, const StepArgs& a,
                                    bool write_u, bool write_rho);
template <typename T>
mlbm_status launch_compact_pass(mlbm_lattice* lat, const StepArgs& a, int pass,
                                bool write_u, bool write_rho);
bool compact_two_pass_supported(int lx, int ly, int lz, int storage);
// Wavefront step over the compact layout (compact.cu, wave.cuh).
template <typename T>
mlbm_status launch_compact_wave(mlbm_lattice* lat, const StepArgs& a,
                                bool write_u, bool write_rho);
mlbm_status compact_set_wave_shape(mlbm_lattice* lat, int tile, int lookahead);
void compact_reset_wave(mlbm_lattice* lat);  // after a failed wait
// One-pass step over the compact layout with two buffers (compact.cu,
// band.cuh); starts and ends in AA phase 1.
template <typename T>
mlbm_status launch_compact_band(mlbm_lattice* lat, const StepArgs& a,
                                bool write_u, bool write_rho);
bool compact_band_supported(const mlbm_lattice* lat, int rows);
mlbm_status compact_set_band_shape(mlbm_lattice* lat, int rows, int planes);
}  // namespace mlbm
