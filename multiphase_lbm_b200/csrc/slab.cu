// slab.cu -- one lattice split along z into slabs (include/mlbm.h, "Slab
// decomposition"): the pass-by-pass step and the halo segments a transport
// (NCCL send/recv between GPUs, or device copies between slabs on one GPU)
// moves between the passes.
//
// Why the halos are what they are (AA pattern, pair.cuh conventions): in
// phase 1 every node reads and writes only its own slots; in phase 0 node x
// reads and writes slot d of its neighbour x + e_d.  So for a slab whose
// upper halo plane H is the next slab's lower own plane E:
//   * phase 0 of the upper own plane touches exactly the slots d with
//     e_z(d) = +1 of H (5 directions).  Before the step they must hold what
//     E's owner wrote there in its phase-1 step (its own slots); after the
//     step they hold what this slab's nodes pushed across the face, which
//     E's owner reads in its next (local) step.  No node of E's owner touches
//     those slots of E in phase 0 (their writers lie below E, in this slab).
//   * the update pass reads psi at x + e_i, one plane beyond the own planes.
// The lower face mirrors this with e_z(d) = -1.  Both passes advance only
// the own planes (compact index range [plane_start[1], plane_start[lz - 1]),
// compact.cu), so the halo planes are never written by the kernels except
// through the pushes above.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/mlbm.h"
#include "capi_internal.h"
#include "errors.h"
#include "lattice.cuh"

using namespace mlbm;

namespace {

mlbm_status slab_cuda(cudaError_t e, const char* where) {
  cudaGetLastError();
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
  return set_error(MLBM_ERR_CUDA, msg);
}

bool two_pass_storage(const mlbm_lattice* lat) {
  return lat->storage == MLBM_STORE_F32 || lat->storage == MLBM_STORE_F16;
}

mlbm_status ready_for_passes(mlbm_lattice* lat, const char* who) {
  char msg[160];
  if (!lat) return set_error(MLBM_ERR_ARG, "null lattice handle");
  if (!lat->initialized) {
    std::snprintf(msg, sizeof msg, "%s before initialize", who);
    return set_error(MLBM_ERR_STATE, msg);
  }
  if (!two_pass_storage(lat) || !lat->compact.two_pass_ok) {
    std::snprintf(msg, sizeof msg,
                  "%s: needs FP32 or FP16 storage and a lattice the compact "
                  "two-pass step supports", who);
    return set_error(MLBM_ERR_ARG, msg);
  }
  cudaError_t e = cudaSetDevice(lat->device);
  if (e != cudaSuccess) return slab_cuda(e, "cudaSetDevice");
  return compact_enter(lat);
}

}  // namespace

extern "C" {

mlbm_status mlbm_set_slab(mlbm_lattice* lat, int32_t enable) {
  if (mlbm_status st = ready_for_passes(lat, "set_slab")) return st;
  if (enable && lat->g.lz < 3)
    return set_error(MLBM_ERR_ARG,
                     "set_slab: a slab needs two halo planes and at least one "
                     "own plane (z-extent >= 3)");
  lat->slab = enable != 0;
  return MLBM_OK;
}

mlbm_status mlbm_step_pass(mlbm_lattice* lat, int64_t step, int32_t pass,
                           int32_t reverse, uint32_t inject_type,
                           uint32_t flags) {
  if (pass != 0 && pass != 1)
    return set_error(MLBM_ERR_ARG, "step_pass: pass must be 0 (density) or 1 (update)");
  if (mlbm_status st = ready_for_passes(lat, "step_pass")) return st;
  const bool wu = pass == 1 && (flags & MLBM_ITER_WRITE_VELOCITY);
  if (wu && !lat->vel) {
    // the velocity field is allocated on first request; solid nodes read 0
    const size_t bytes = (size_t)lat->g.plane * 3 * sizeof(float);
    cudaError_t e = cudaMalloc((void**)&lat->vel, bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(lat->vel, 0, bytes, lat->stream);
    if (e != cudaSuccess) return slab_cuda(e, "velocity allocation");
  }
  const StepArgs a{(long long)step, reverse, inject_type};
  mlbm_status st;
  if (lat->storage == MLBM_STORE_F32)
    st = launch_compact_pass<float>(lat, a, pass, wu, pass == 0);
  else
    st = launch_compact_pass<__half>(lat, a, pass, wu, pass == 0);
  if (st) return st;
  lat->compact.parts_valid = false;
  if (pass == 1) {
    lat->phase ^= 1;
    if (wu) lat->vel_valid = true;
  }
  return MLBM_OK;
}

mlbm_status mlbm_halo_segments(mlbm_lattice* lat, int32_t kind, int32_t side,
                               void** ptrs, int64_t* bytes, int32_t* count) {
  if (!ptrs || !bytes || !count)
    return set_error(MLBM_ERR_ARG, "halo_segments: null output");
  if (side != 0 && side != 1)
    return set_error(MLBM_ERR_ARG, "halo_segments: side must be 0 or 1");
  if (mlbm_status st = ready_for_passes(lat, "halo_segments")) return st;
  if (!lat->slab)
    return set_error(MLBM_ERR_STATE, "halo_segments: not a slab lattice");
  const Geom& g = lat->g;
  const CompactState& c = lat->compact;
  const bool edge = kind == MLBM_HALO_PSI_EDGE || kind == MLBM_HALO_POP_EDGE;
  // edge planes: 1 (lower face) and lz - 2 (upper); halo planes: 0 and lz - 1
  const int z = edge ? (side == 0 ? 1 : g.lz - 2) : (side == 0 ? 0 : g.lz - 1);
  if (kind == MLBM_HALO_PSI_EDGE || kind == MLBM_HALO_PSI_GHOST) {
    // one padded psi plane, ghost columns and rows included
    const long long plane = (long long)(g.ly + 2) * g.pxg;
    ptrs[0] = static_cast<float*>(lat->psi) + psi_index(g, -4, -1, z);
    bytes[0] = plane * (long long)sizeof(float);
    *count = 1;
    return MLBM_OK;
  }
  if (kind != MLBM_HALO_POP_EDGE && kind != MLBM_HALO_POP_GHOST)
    return set_error(MLBM_ERR_ARG, "halo_segments: unknown kind");
  // the slots streamed across the face: e_z = +1 across the upper face of
  // the slab below (its halo side 1 = this slab's edge side 0), e_z = -1
  // across the lower face
  const int dir = (edge ? side == 0 : side == 1) ? 1 : -1;
  const size_t elem = pop_elem_bytes(lat->storage);
  const long long k0 = c.plane_start[z], n = c.plane_start[z + 1] - k0;
  int m = 0;
  for (int d = 1; d < Q; ++d) {
    if (ez(d) != dir) continue;
    ptrs[m] = static_cast<char*>(c.cpop) + ((long long)d * c.cs + k0) * (long long)elem;
    bytes[m] = n * (long long)elem;
    ++m;
  }
  *count = m;
  return MLBM_OK;
}

}  // extern "C"
