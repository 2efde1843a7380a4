// capi_internal.h -- the lattice handle behind the C ABI (not exported).
#pragma once

#include <cuda_runtime.h>

#include "../../include/mlbm.h"
#include "errors.h"
#include "lattice.cuh"

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
  float* vel = nullptr;         // [node][3], written on request
  void* staging = nullptr;      // reference-layout transfer buffer
  size_t staging_bytes = 0;
  double* stats_scratch = nullptr;
  size_t stats_scratch_bytes = 0;

  int phase = 0;  // 0: post-collision at opp slots of own node; 1: pushed
  bool has_params = false, has_mask = false, has_rho = false;
  bool initialized = false;
  bool vel_valid = false;
};

namespace mlbm {
mlbm_status cuda_fail(cudaError_t e, const char* where);
size_t pop_elem_bytes(int storage);
size_t real_bytes(int storage);
Geom make_geom(int lx, int ly, int lz);
}  // namespace mlbm
