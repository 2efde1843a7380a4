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

#include <algorithm>
#include <cstdio>
#include <vector>

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

// Segments of one halo kind on one side of a slab lattice whose compact
// layout is active: pointers, byte sizes and (population kinds) the direction
// of each segment; returns the segment count.
int halo_segs(const mlbm_lattice* lat, int kind, int side, void** ptrs,
              int64_t* bytes, int* dirs) {
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
    dirs[0] = 0;
    return 1;
  }
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
    dirs[m] = d;
    ++m;
  }
  return m;
}

// ---- in-process ring exchange: one kernel per exchange -----------------------
// One copy job per halo segment: dst[k] = src[k] for k < count, or, with
// dst_info (the receiving edge plane's node words), only where bit `bit` of
// the node word is set (the pusher y - e_bit is fluid).
struct HaloJob {
  const void* src;
  void* dst;
  const uint2* dst_info;
  int count;
  int bit;
};

template <typename E>
__global__ void k_halo_jobs(const HaloJob* __restrict__ jobs) {
  const HaloJob j = jobs[blockIdx.y];
  const E* __restrict__ src = static_cast<const E*>(j.src);
  E* __restrict__ dst = static_cast<E*>(j.dst);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < j.count;
       k += gridDim.x * blockDim.x) {
    if (j.dst_info && !((j.dst_info[k].x >> j.bit) & 1u)) continue;
    dst[k] = src[k];
  }
}

constexpr int kRingKinds = 3;

}  // namespace

struct mlbm_slab_ring {
  int device = 0;
  int elem = 4;  // population element bytes (psi: always 4)
  std::vector<mlbm_lattice*> slabs;
  HaloJob* jobs[kRingKinds] = {nullptr, nullptr, nullptr};
  int njobs[kRingKinds] = {0, 0, 0};
  int maxcount[kRingKinds] = {0, 0, 0};
  std::vector<cudaEvent_t> ready;  // per slab: its stream reached the exchange
  cudaEvent_t done = nullptr;
};

namespace {

void ring_free(mlbm_slab_ring* r) {
  for (HaloJob*& j : r->jobs) {
    if (j) cudaFree(j);
    j = nullptr;
  }
  for (cudaEvent_t e : r->ready)
    if (e) cudaEventDestroy(e);
  if (r->done) cudaEventDestroy(r->done);
  delete r;
}

// The jobs of one exchange kind: for every slab i, the moves of its two
// faces (slab.py, MOVES_IN / MOVES_OUT): side 1 to slab i + 1's side 0 and
// side 0 to slab i - 1's side 1.
bool ring_jobs(const mlbm_slab_ring* r, int what, std::vector<HaloJob>& out,
               int& maxcount) {
  const int n = (int)r->slabs.size();
  const int src_kind = what == MLBM_RING_POP_IN ? MLBM_HALO_POP_EDGE
                       : what == MLBM_RING_PSI  ? MLBM_HALO_PSI_EDGE
                                                : MLBM_HALO_POP_GHOST;
  const int dst_kind = what == MLBM_RING_POP_IN ? MLBM_HALO_POP_GHOST
                       : what == MLBM_RING_PSI  ? MLBM_HALO_PSI_GHOST
                                                : MLBM_HALO_POP_EDGE;
  const int elem = what == MLBM_RING_PSI ? 4 : r->elem;
  maxcount = 0;
  for (int i = 0; i < n; ++i) {
    for (int m = 0; m < 2; ++m) {
      const int src_side = m == 0 ? 1 : 0, dst_side = 1 - src_side;
      const mlbm_lattice* a = r->slabs[i];
      const mlbm_lattice* b = r->slabs[(i + (m == 0 ? 1 : n - 1)) % n];
      void* sp[MLBM_HALO_MAX_SEGMENTS];
      void* dp[MLBM_HALO_MAX_SEGMENTS];
      int64_t sb[MLBM_HALO_MAX_SEGMENTS], db[MLBM_HALO_MAX_SEGMENTS];
      int sd[MLBM_HALO_MAX_SEGMENTS], dd[MLBM_HALO_MAX_SEGMENTS];
      const int ns = halo_segs(a, src_kind, src_side, sp, sb, sd);
      // receiving edge plane (merge): its first compact node
      const int zb = dst_side == 0 ? 1 : b->g.lz - 2;
      const uint2* info = b->compact.cinfo + b->compact.plane_start[zb];
      const int nd = halo_segs(b, dst_kind, dst_side, dp, db, dd);
      if (nd != ns) return false;
      for (int k = 0; k < ns; ++k) {
        if (sb[k] != db[k] || sd[k] != dd[k]) return false;  // not the same plane
        if (sb[k] == 0) continue;
        HaloJob j;
        j.src = sp[k];
        j.dst = dp[k];
        j.dst_info = what == MLBM_RING_POP_OUT ? info : nullptr;
        j.count = (int)(sb[k] / elem);
        j.bit = dd[k];
        out.push_back(j);
        maxcount = std::max(maxcount, j.count);
      }
    }
  }
  return true;
}

}  // namespace

extern "C" {

mlbm_status mlbm_set_slab(mlbm_lattice* lat, int32_t enable) {
  DeviceGuard restore_device;
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
  DeviceGuard restore_device;
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
  if (pass == 1) {
    lat->phase ^= 1;
    if (wu) lat->vel_valid = true;
  }
  return MLBM_OK;
}

mlbm_status mlbm_halo_segments(mlbm_lattice* lat, int32_t kind, int32_t side,
                               void** ptrs, int64_t* bytes, int32_t* count) {
  DeviceGuard restore_device;
  if (!ptrs || !bytes || !count)
    return set_error(MLBM_ERR_ARG, "halo_segments: null output");
  if (side != 0 && side != 1)
    return set_error(MLBM_ERR_ARG, "halo_segments: side must be 0 or 1");
  if (kind < MLBM_HALO_PSI_EDGE || kind > MLBM_HALO_POP_GHOST)
    return set_error(MLBM_ERR_ARG, "halo_segments: unknown kind");
  if (mlbm_status st = ready_for_passes(lat, "halo_segments")) return st;
  if (!lat->slab)
    return set_error(MLBM_ERR_STATE, "halo_segments: not a slab lattice");
  int dirs[MLBM_HALO_MAX_SEGMENTS];
  *count = halo_segs(lat, kind, side, ptrs, bytes, dirs);
  return MLBM_OK;
}


mlbm_status mlbm_slab_ring_create(mlbm_lattice* const* slabs, int32_t n,
                                  mlbm_slab_ring** out) {
  DeviceGuard restore_device;
  if (!slabs || n < 1 || !out)
    return set_error(MLBM_ERR_ARG, "slab_ring_create: bad arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (mlbm_status st = ready_for_passes(slabs[i], "slab_ring_create")) return st;
    if (!slabs[i]->slab)
      return set_error(MLBM_ERR_STATE, "slab_ring_create: not a slab lattice");
    if (slabs[i]->storage != slabs[0]->storage || slabs[i]->g.lx != slabs[0]->g.lx ||
        slabs[i]->g.ly != slabs[0]->g.ly)
      return set_error(MLBM_ERR_ARG,
                       "slab_ring_create: slabs differ in storage or x-y extent");
  }
  mlbm_slab_ring* r = new mlbm_slab_ring();
  r->device = slabs[0]->device;
  r->elem = (int)pop_elem_bytes(slabs[0]->storage);
  r->slabs.assign(slabs, slabs + n);
  cudaError_t e = cudaSetDevice(r->device);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    const int d = slabs[i]->device;
    if (d == r->device) continue;
    int ok = 0;
    e = cudaDeviceCanAccessPeer(&ok, r->device, d);
    if (e == cudaSuccess && !ok) {
      ring_free(r);
      return set_error(MLBM_ERR_ARG, "slab_ring_create: no peer access between the slabs' GPUs");
    }
    if (e == cudaSuccess) {
      e = cudaDeviceEnablePeerAccess(d, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) {
        cudaGetLastError();
        e = cudaSuccess;
      }
    }
  }
  for (int w = 0; w < kRingKinds && e == cudaSuccess; ++w) {
    std::vector<HaloJob> jobs;
    if (!ring_jobs(r, w, jobs, r->maxcount[w])) {
      ring_free(r);
      return set_error(MLBM_ERR_ARG,
                       "slab_ring_create: neighbouring slabs' halo and edge "
                       "planes differ (slabs not cut from one lattice in z order)");
    }
    r->njobs[w] = (int)jobs.size();
    if (jobs.empty()) continue;
    e = cudaMalloc((void**)&r->jobs[w], jobs.size() * sizeof(HaloJob));
    if (e == cudaSuccess)
      e = cudaMemcpy(r->jobs[w], jobs.data(), jobs.size() * sizeof(HaloJob),
                     cudaMemcpyHostToDevice);
  }
  r->ready.assign(n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaSetDevice(slabs[i]->device);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->ready[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaSetDevice(r->device);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ring_free(r);
    return slab_cuda(e, "slab_ring_create");
  }
  *out = r;
  return MLBM_OK;
}

mlbm_status mlbm_slab_ring_exchange(mlbm_slab_ring* r, int32_t what) {
  DeviceGuard restore_device;
  if (!r) return set_error(MLBM_ERR_ARG, "slab_ring_exchange: null ring");
  if (what < 0 || what >= kRingKinds)
    return set_error(MLBM_ERR_ARG, "slab_ring_exchange: unknown exchange");
  cudaStream_t s0 = r->slabs[0]->stream;
  cudaError_t e = cudaSuccess;
  const int n = (int)r->slabs.size();
  // the kernel runs on slab 0's stream after every slab's pending work
  for (int i = 1; i < n && e == cudaSuccess; ++i) {
    mlbm_lattice* l = r->slabs[i];
    if (l->device == r->device && l->stream == s0) continue;
    e = cudaSetDevice(l->device);
    if (e == cudaSuccess) e = cudaEventRecord(r->ready[i], l->stream);
    if (e == cudaSuccess) e = cudaSetDevice(r->device);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s0, r->ready[i], 0);
  }
  if (e == cudaSuccess) e = cudaSetDevice(r->device);
  if (e == cudaSuccess && r->njobs[what] > 0) {
    const int threads = 256;
    const int gx = std::max(1, std::min((r->maxcount[what] + threads - 1) / threads, 64));
    const dim3 grid(gx, r->njobs[what]);
    if (what == MLBM_RING_PSI || r->elem == 4)
      k_halo_jobs<uint32_t><<<grid, threads, 0, s0>>>(r->jobs[what]);
    else
      k_halo_jobs<uint16_t><<<grid, threads, 0, s0>>>(r->jobs[what]);
    e = cudaGetLastError();
  }
  // and every slab's later work runs after it
  bool others = false;
  for (int i = 1; i < n; ++i)
    others |= r->slabs[i]->device != r->device || r->slabs[i]->stream != s0;
  if (e == cudaSuccess && others) e = cudaEventRecord(r->done, s0);
  for (int i = 1; i < n && e == cudaSuccess && others; ++i) {
    mlbm_lattice* l = r->slabs[i];
    if (l->device == r->device && l->stream == s0) continue;
    e = cudaSetDevice(l->device);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(l->stream, r->done, 0);
  }
  if (e == cudaSuccess) e = cudaSetDevice(r->device);
  if (e != cudaSuccess) return slab_cuda(e, "slab_ring_exchange");
  return MLBM_OK;
}

mlbm_status mlbm_slab_ring_destroy(mlbm_slab_ring* r) {
  DeviceGuard restore_device;
  if (!r) return MLBM_OK;
  cudaSetDevice(r->device);
  ring_free(r);
  return MLBM_OK;
}

}  // extern "C"
