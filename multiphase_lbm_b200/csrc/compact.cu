// compact.cu -- host side of the single-pass step over the compact layout
// (compact.cuh): tables built from the mask, tiling, layout changes, launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "capi_internal.h"
#include "compact.cuh"
#include "band.cuh"
#include "compact2.cuh"
#include "wave.cuh"

namespace mlbm {

namespace {

dim3 node_block() { return dim3(32, 4, 1); }
dim3 node_grid(const Geom& g) { return dim3(g.px / 32, (g.ly + 3) / 4, g.lz); }

constexpr size_t kSmemMax = 227 * 1024;

// Part buffers: two sets of [4][cs]; a step from AA phase `ph` reads set ph
// and writes set ph ^ 1 (the phase alternates with every step).
CArgs args_of(const mlbm_lattice* lat) {
  const CompactState& c = lat->compact;
  const Geom& g = lat->g;
  const int ph = lat->phase;
  CArgs a;
  a.mask = lat->mask;
  a.wbase = c.wbase;
  a.cnb = c.cnb;
  a.ytab = c.tabs;
  a.ztab = c.tabs + g.ly;
  a.ystart = c.tabs + g.ly + g.lz;
  a.zstart = c.tabs + g.ly + g.lz + (c.nty + 1);
  a.part_rd = c.part + (size_t)ph * 4 * c.cs;
  a.part_wr = c.part + (size_t)(ph ^ 1) * 4 * c.cs;
  a.cs = c.cs;
  a.nty = c.nty;
  a.nzc = c.nzc;
  a.rows_max = c.rows_max;
  return a;
}

// Split n into k nearly equal parts (each at least 2 when n >= 2k).
std::vector<int> split(int n, int k) {
  std::vector<int> s(k + 1);
  for (int i = 0; i <= k; ++i) s[i] = (int)((long long)i * n / k);
  return s;
}

// Tiles of `rows` rows along y and chunks of `planes` planes along z; at
// least two of each, each at least two rows / planes.
mlbm_status build_tiling(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  const Geom& g = lat->g;
  const int nty = std::max(2, std::min(g.ly / 2, g.ly / std::max(1, c.rows)));
  const int nzc = std::max(2, std::min(g.lz / 2, g.lz / std::max(1, c.planes)));
  const std::vector<int> ys = split(g.ly, nty), zs = split(g.lz, nzc);
  int rows_max = 0;
  for (int t = 0; t < nty; ++t) rows_max = std::max(rows_max, ys[t + 1] - ys[t]);
  const size_t smem = compact_smem_bytes(rows_max, g.lx, g.wpr);
  if (smem > kSmemMax)
    return set_error(MLBM_ERR_ARG, "compact step: tile does not fit shared memory");
  std::vector<int> tab(g.ly + g.lz + nty + 1 + nzc + 1);
  for (int t = 0; t < nty; ++t)
    for (int y = ys[t]; y < ys[t + 1]; ++y)
      tab[y] = t | (y == ys[t] ? kEdgeLo : 0) | (y == ys[t + 1] - 1 ? kEdgeHi : 0);
  for (int t = 0; t < nzc; ++t)
    for (int z = zs[t]; z < zs[t + 1]; ++z)
      tab[g.ly + z] =
          t | (z == zs[t] ? kEdgeLo : 0) | (z == zs[t + 1] - 1 ? kEdgeHi : 0);
  std::copy(ys.begin(), ys.end(), tab.begin() + g.ly + g.lz);
  std::copy(zs.begin(), zs.end(), tab.begin() + g.ly + g.lz + nty + 1);
  if (c.tabs) cudaFree(c.tabs);
  c.tabs = nullptr;
  cudaError_t e = cudaMalloc((void**)&c.tabs, tab.size() * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(c.tabs, tab.data(), tab.size() * sizeof(int),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "compact tiling tables");
  c.nty = nty;
  c.nzc = nzc;
  c.rows_max = rows_max;
  c.smem = smem;
  return MLBM_OK;
}

// Fluid counts per mask word, scanned into wbase; buffers for the fluid
// nodes.
mlbm_status build_tables(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  const Geom& g = lat->g;
  const long long nwords = (long long)g.lz * g.ly * g.wpr;
  cudaError_t e = cudaStreamSynchronize(lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact tables");
  if (c.wbase) cudaFree(c.wbase);
  c.wbase = nullptr;
  e = cudaMalloc((void**)&c.wbase, (nwords + 1) * sizeof(uint32_t));
  if (e != cudaSuccess) return cuda_fail(e, "compact tables");
  k_word_counts<<<(unsigned)((nwords + 255) / 256), 256, 0, lat->stream>>>(
      lat->mask, c.wbase, nwords);
  std::vector<uint32_t> h(nwords + 1);
  e = cudaMemcpyAsync(h.data(), c.wbase, nwords * sizeof(uint32_t),
                      cudaMemcpyDeviceToHost, lat->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact tables");
  // every plane starts at an even compact index: a plane with an odd fluid
  // count is followed by one unused slot (a hole), so node pairs (pair.cuh)
  // never straddle two planes
  unsigned long long run = 0;
  const long long words_per_plane = (long long)g.ly * g.wpr;
  for (long long i = 0; i < nwords; ++i) {
    if (i > 0 && i % words_per_plane == 0) run += run & 1ull;
    const uint32_t v = h[i];
    h[i] = (uint32_t)run;
    run += v;
  }
  run += run & 1ull;
  h[nwords] = (uint32_t)run;
  if (run >= (1ull << 31))
    return set_error(MLBM_ERR_ARG, "compact step: more than 2^31 fluid nodes");
  c.plane_start.assign(g.lz + 1, 0);
  for (int z = 0; z <= g.lz; ++z)
    c.plane_start[z] = h[(long long)z * g.ly * g.wpr];
  c.wave_built = false;
  e = cudaMemcpy(c.wbase, h.data(), (nwords + 1) * sizeof(uint32_t),
                 cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "compact tables");
  if (c.wtab) cudaFree(c.wtab);
  c.wtab = nullptr;
  e = cudaMalloc((void**)&c.wtab, (nwords + 1) * sizeof(uint2));
  if (e != cudaSuccess) return cuda_fail(e, "compact tables");
  k_wtab<<<(unsigned)((nwords + 256) / 256), 256, 0, lat->stream>>>(
      lat->mask, c.wbase, c.wtab, nwords);
  c.nfluid = (long long)run;  // compact slots: fluid nodes and holes
  c.cs = std::max(64LL, (c.nfluid + 63) / 64 * 64);
  if (c.cs > c.cap) {
    cudaFree(c.cpop);
    cudaFree(c.cpop_alt);
    c.cpop_alt = nullptr;
    cudaFree(c.part);
    cudaFree(c.cnb);
    cudaFree(c.cinfo);
    c.cpop = nullptr;
    c.part = nullptr;
    c.cnb = nullptr;
    c.cinfo = nullptr;
    c.cap = 0;
    e = cudaMalloc(&c.cpop, (size_t)c.cs * Q * pop_elem_bytes(lat->storage));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c.part, (size_t)c.cs * 8 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c.cnb, (size_t)c.cs * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c.cinfo, (size_t)c.cs * sizeof(uint2));
    if (e != cudaSuccess) {
      cudaFree(c.cpop);
      cudaFree(c.part);
      cudaFree(c.cnb);
      c.cpop = nullptr;
      c.part = nullptr;
      c.cnb = nullptr;
      cudaGetLastError();
      return cuda_fail(e, "compact buffers");
    }
    c.cap = c.cs;
  }
  if (mlbm_status st = build_tiling(lat)) return st;
  c.built = true;
  return MLBM_OK;
}

template <typename T>
mlbm_status enter_t(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  // the seed goes to the set the next step reads (set `phase`)
  CArgs a = args_of(lat);
  float* seed = c.part + (size_t)lat->phase * 4 * c.cs;
  a.part_wr = seed;
  k_convert<T, true><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<T*>(lat->pop), static_cast<T*>(c.cpop), lat->nbw, c.cnb, a,
      lat->g);
  // holes keep (0, 0): no fluid bit
  cudaError_t e = cudaMemsetAsync(c.cinfo, 0, c.cs * sizeof(uint2), lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact node table");
  k_cinfo<<<node_grid(lat->g), node_block(), 0, lat->stream>>>(lat->nbw, c.cinfo,
                                                                a, lat->g);
  e = cudaMemsetAsync(seed + c.cs, 0, 3 * c.cs * sizeof(float), lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact parts");
  if (lat->phase == 0)
    k_seed_parts<T, 0><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        static_cast<const T*>(lat->pop), lat->nbw, a, lat->g, lat->phys);
  else
    k_seed_parts<T, 1><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        static_cast<const T*>(lat->pop), lat->nbw, a, lat->g, lat->phys);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact entry launch");
  return MLBM_OK;
}

template <typename T>
mlbm_status to_dense_t(mlbm_lattice* lat) {
  const CArgs a = args_of(lat);
  k_convert<T, false><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<T*>(lat->pop), static_cast<T*>(lat->compact.cpop), nullptr,
      nullptr, a, lat->g);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact exit launch");
  return MLBM_OK;
}

template <typename T, int PHASE, int OUT>
const void* step_fn() {
  return reinterpret_cast<const void*>(&k_compact_step<T, PHASE, OUT>);
}

template <typename T>
const void* pick_step(int phase, int out) {
  if (phase == 0) {
    switch (out) {
      case OUT_NONE: return step_fn<T, 0, OUT_NONE>();
      case OUT_RHO: return step_fn<T, 0, OUT_RHO>();
      default: return step_fn<T, 0, OUT_RHO | OUT_VEL>();
    }
  }
  switch (out) {
    case OUT_NONE: return step_fn<T, 1, OUT_NONE>();
    case OUT_RHO: return step_fn<T, 1, OUT_RHO>();
    default: return step_fn<T, 1, OUT_RHO | OUT_VEL>();
  }
}

template <typename T>
mlbm_status set_smem_attr(size_t smem) {
  for (int ph = 0; ph < 2; ++ph)
    for (int out : {(int)OUT_NONE, (int)OUT_RHO, (int)(OUT_RHO | OUT_VEL)}) {
      cudaError_t e = cudaFuncSetAttribute(pick_step<T>(ph, out),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return cuda_fail(e, "compact step attribute");
    }
  return MLBM_OK;
}

}  // namespace

bool compact_supported(int lx, int ly, int lz, int storage) {
  if (storage == MLBM_STORE_F64) return false;
  if (ly < 4 || lz < 4 || lx > 65535) return false;
  const Geom g = make_geom(lx, ly, lz);
  return compact_smem_bytes(2, lx, g.wpr) <= kSmemMax;
}

// Population offsets of the compact kernels are 32-bit (pair.cuh):
// Q * cs < 2^32 holds for every lattice of fewer than kC2MaxNodes nodes.
// (margin: up to one hole per plane and the rounding of cs to 64)
constexpr long long kC2MaxNodes = (1LL << 32) / Q - 4096;

bool compact_two_pass_supported(int lx, int ly, int lz, int storage) {
  return storage != MLBM_STORE_F64 && lx <= kC2MaxX && ly <= kC2MaxY &&
         lz <= kC2MaxZ && (long long)lx * ly * lz <= kC2MaxNodes;
}

mlbm_status compact_set_shape(mlbm_lattice* lat, int rows, int planes) {
  CompactState& c = lat->compact;
  const int old_rows = c.rows, old_planes = c.planes;
  c.rows = rows;
  c.planes = planes;
  if (!c.built) return MLBM_OK;
  if (mlbm_status st = build_tiling(lat)) {
    c.rows = old_rows;
    c.planes = old_planes;
    build_tiling(lat);
    return st;
  }
  // the parts of the last step follow the old tiling: take them again from
  // the populations
  if (c.active) {
    if (mlbm_status st = compact_leave(lat)) return st;
    return compact_enter(lat);
  }
  return MLBM_OK;
}

mlbm_status compact_enter(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  if (c.active) return MLBM_OK;
  if (!c.supported && !c.two_pass_ok)
    return set_error(MLBM_ERR_ARG, "compact layout does not support this lattice");
  if (!c.built)
    if (mlbm_status st = build_tables(lat)) return st;
  mlbm_status st;
  switch (lat->storage) {
    case MLBM_STORE_F32: st = enter_t<float>(lat); break;
    default: st = enter_t<__half>(lat); break;
  }
  if (st) return st;
  c.active = true;
  c.parts_valid = true;
  return MLBM_OK;
}

mlbm_status compact_sync_dense(mlbm_lattice* lat) {
  if (!lat->compact.active) return MLBM_OK;
  switch (lat->storage) {
    case MLBM_STORE_F32: return to_dense_t<float>(lat);
    default: return to_dense_t<__half>(lat);
  }
}

mlbm_status compact_leave(mlbm_lattice* lat) {
  if (!lat->compact.active) return MLBM_OK;
  if (mlbm_status st = compact_sync_dense(lat)) return st;
  lat->compact.active = false;
  return MLBM_OK;
}

void compact_invalidate(mlbm_lattice* lat) {
  lat->compact.built = false;
  lat->compact.active = false;
}

void compact_free(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  cudaFree(c.cpop);
  cudaFree(c.cpop_alt);
  cudaFree(c.part);
  cudaFree(c.cnb);
  cudaFree(c.cinfo);
  cudaFree(c.wbase);
  cudaFree(c.wtab);
  cudaFree(c.tabs);
  cudaFree(c.wave_items);
  cudaFree(c.wave_need);
  cudaFree(c.wave_ctl);
  c = CompactState{};
}

// The dynamic shared-memory limit is an attribute of the kernel on each
// device: raise it (never lower it) to the largest size any lattice needs.
template <typename T>
mlbm_status ensure_smem_attr(int device, size_t smem) {
  constexpr int kDevices = 64;
  static std::mutex mu;
  static size_t granted[kDevices] = {};
  if (device < 0 || device >= kDevices)
    return set_error(MLBM_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (granted[device] >= smem) return MLBM_OK;
  if (mlbm_status st = set_smem_attr<T>(smem)) return st;
  granted[device] = smem;
  return MLBM_OK;
}

template <typename T>
mlbm_status launch_compact(mlbm_lattice* lat, const StepArgs& a, int out) {
  CompactState& c = lat->compact;
  if (mlbm_status st = ensure_smem_attr<T>(lat->device, c.smem)) return st;
  T* cpop = static_cast<T*>(c.cpop);
  float* rho = static_cast<float*>(lat->rho);
  float* psi = static_cast<float*>(lat->psi);
  float* vel = lat->vel;
  Geom g = lat->g;
  Phys p = lat->phys;
  StepArgs aa = a;
  CArgs cc = args_of(lat);
  void* args[] = {&cpop, &cc, &rho, &psi, &vel, &g, &p, &aa};
  cudaError_t e = cudaLaunchKernel(pick_step<T>(lat->phase, out),
                                   dim3(c.nty * c.nzc), dim3(kCompactThreads), args,
                                   c.smem, lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact time-step launch");
  return MLBM_OK;
}

template mlbm_status launch_compact<float>(mlbm_lattice*, const StepArgs&, int);
template mlbm_status launch_compact<__half>(mlbm_lattice*, const StepArgs&, int);

namespace {
// Compact indices the step advances: all fluid nodes, or for a slab lattice
// the planes between its two halo planes.
void own_range(const mlbm_lattice* lat, long long& kb, long long& ke) {
  const CompactState& c = lat->compact;
  if (lat->slab) {
    kb = c.plane_start[1];
    ke = c.plane_start[lat->g.lz - 1];
  } else {
    kb = 0;
    ke = c.nfluid;
  }
}

unsigned c2_grid(long long kb, long long ke, long long per_thread) {
  const long long threads = (ke - kb + per_thread - 1) / per_thread;
  return (unsigned)((threads + kC2Threads - 1) / kC2Threads);
}

template <typename T, int PHASE>
void launch_c2_density(mlbm_lattice* lat, const StepArgs& a, bool wr, bool inj) {
  const CompactState& c = lat->compact;
  long long kb, ke;
  own_range(lat, kb, ke);
  const unsigned grid = c2_grid(kb, ke, c2_nodes_per_thread<PHASE>());
  if (grid == 0) return;
  const T* cpop = static_cast<const T*>(c.cpop);
  const uint32_t cs = (uint32_t)c.cs;
  float* rho = static_cast<float*>(lat->rho);
  float* psi = static_cast<float*>(lat->psi);
  if (wr)
    k_cdensity<T, PHASE, true><<<grid, kC2Threads, 0, lat->stream>>>(
        cpop, cs, c.cinfo, c.wtab, (int)kb, (int)ke, rho, psi, lat->g, lat->phys,
        a, inj);
  else
    k_cdensity<T, PHASE, false><<<grid, kC2Threads, 0, lat->stream>>>(
        cpop, cs, c.cinfo, c.wtab, (int)kb, (int)ke, rho, psi, lat->g, lat->phys,
        a, inj);
}

template <typename T, int PHASE>
void launch_c2_update(mlbm_lattice* lat, const StepArgs& a, bool wu, bool inj) {
  const CompactState& c = lat->compact;
  long long kb, ke;
  own_range(lat, kb, ke);
  const unsigned grid = c2_grid(kb, ke, c2_nodes_per_thread<PHASE>());
  if (grid == 0) return;
  T* cpop = static_cast<T*>(c.cpop);
  const uint32_t cs = (uint32_t)c.cs;
  const float* psi = static_cast<const float*>(lat->psi);
  if (wu)
    k_cupdate<T, PHASE, true><<<grid, kC2Threads, 0, lat->stream>>>(
        cpop, cs, c.cinfo, c.wtab, (int)kb, (int)ke, psi, lat->vel, lat->g,
        lat->phys, a, inj);
  else
    k_cupdate<T, PHASE, false><<<grid, kC2Threads, 0, lat->stream>>>(
        cpop, cs, c.cinfo, c.wtab, (int)kb, (int)ke, psi, lat->vel, lat->g,
        lat->phys, a, inj);
}

bool inject_now(const mlbm_lattice* lat, const StepArgs& a) {
  const Phys& p = lat->phys;
  return p.rho_inject_period != 0ull &&
         (unsigned long long)a.step % p.rho_inject_period == 0ull;
}
}  // namespace

template <typename T>
mlbm_status launch_compact_two_pass(mlbm_lattice* lat, const StepArgs& a,
                                    bool write_u, bool write_rho) {
  const bool inj = inject_now(lat, a);
  if (lat->phase == 0) {
    launch_c2_density<T, 0>(lat, a, write_rho, inj);
    launch_c2_update<T, 0>(lat, a, write_u, inj);
  } else {
    launch_c2_density<T, 1>(lat, a, write_rho, inj);
    launch_c2_update<T, 1>(lat, a, write_u, inj);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact two-pass launch");
  return MLBM_OK;
}

template mlbm_status launch_compact_two_pass<float>(mlbm_lattice*, const StepArgs&, bool, bool);
template mlbm_status launch_compact_two_pass<__half>(mlbm_lattice*, const StepArgs&, bool, bool);

// One pass of the compact two-pass step (0: density, 1: update) in the
// lattice's current AA phase; the caller flips the phase after the update.
template <typename T>
mlbm_status launch_compact_pass(mlbm_lattice* lat, const StepArgs& a, int pass,
                                bool write_u, bool write_rho) {
  const bool inj = inject_now(lat, a);
  if (pass == 0) {
    if (lat->phase == 0) launch_c2_density<T, 0>(lat, a, write_rho, inj);
    else launch_c2_density<T, 1>(lat, a, write_rho, inj);
  } else {
    if (lat->phase == 0) launch_c2_update<T, 0>(lat, a, write_u, inj);
    else launch_c2_update<T, 1>(lat, a, write_u, inj);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact pass launch");
  return MLBM_OK;
}

template mlbm_status launch_compact_pass<float>(mlbm_lattice*, const StepArgs&, int, bool, bool);
template mlbm_status launch_compact_pass<__half>(mlbm_lattice*, const StepArgs&, int, bool, bool);

// ---- wavefront step (wave.cuh) ------------------------------------------------

namespace {

// Polls of a waiting update tile before it gives up (a poll is three acquire
// loads and a 64 ns sleep, so the wait ends within about a second).
constexpr unsigned kWaveSpinLimit = 1u << 20;

template <typename T, int PHASE, int OUT>
const void* wave_fn() {
  return reinterpret_cast<const void*>(&k_cwave<T, PHASE, OUT>);
}

template <typename T>
const void* pick_wave(int phase, int out) {
  if (phase == 0) {
    switch (out) {
      case OUT_NONE: return wave_fn<T, 0, OUT_NONE>();
      case OUT_RHO: return wave_fn<T, 0, OUT_RHO>();
      default: return wave_fn<T, 0, OUT_RHO | OUT_VEL>();
    }
  }
  switch (out) {
    case OUT_NONE: return wave_fn<T, 1, OUT_NONE>();
    case OUT_RHO: return wave_fn<T, 1, OUT_RHO>();
    default: return wave_fn<T, 1, OUT_RHO | OUT_VEL>();
  }
}

// Work list of the wavefront: tiles of `tile` fluid nodes that never straddle
// a plane, density tiles `lookahead` planes ahead of the update tiles (the
// order is described in wave.cuh).  Every update tile's dependencies (density
// of planes z-1, z, z+1) come earlier in the list.
mlbm_status build_wave(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  const int lz = lat->g.lz;
  const int tile = (c.wave_tile + 1) & ~1, L = c.wave_lookahead;  // whole pairs
  std::vector<int4> items;
  std::vector<unsigned> need(lz, 0u);
  items.reserve((size_t)(2 * c.nfluid / tile + 2 * lz + 8));
  std::vector<bool> emitted(lz, false);
  auto emit = [&](int z, int kind) {
    for (long long k0 = c.plane_start[z]; k0 < c.plane_start[z + 1]; k0 += tile) {
      const long long k1 = std::min(k0 + tile, c.plane_start[z + 1]);
      items.push_back(make_int4(z, kind, (int)k0, (int)k1));
      if (kind == kWaveDensity) ++need[z];
    }
  };
  auto emit_d = [&](int z) {
    if (z < 0 || z >= lz || emitted[z]) return;
    emitted[z] = true;
    emit(z, kWaveDensity);
  };
  emit_d(lz - 1);
  for (int z = 0; z <= L; ++z) emit_d(z);
  for (int z = 0; z < lz; ++z) {
    emit_d(z + 1);  // already emitted unless lookahead < 1
    emit(z, kWaveUpdate);
    emit_d(z + L + 1);
  }
  if (items.size() > (size_t)INT32_MAX)
    return set_error(MLBM_ERR_ARG, "wavefront step: too many work items");
  cudaError_t e = cudaStreamSynchronize(lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wavefront work list");
  cudaFree(c.wave_items);
  cudaFree(c.wave_need);
  cudaFree(c.wave_ctl);
  c.wave_items = nullptr;
  c.wave_need = nullptr;
  c.wave_ctl = nullptr;
  e = cudaMalloc((void**)&c.wave_items, std::max<size_t>(1, items.size()) * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c.wave_need, lz * sizeof(unsigned));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&c.wave_ctl, (2 + 2 * (size_t)lz) * sizeof(unsigned));
  if (e == cudaSuccess && !items.empty())
    e = cudaMemcpy(c.wave_items, items.data(), items.size() * sizeof(int4),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c.wave_need, need.data(), lz * sizeof(unsigned),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemset(c.wave_ctl, 0, (2 + 2 * (size_t)lz) * sizeof(unsigned));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cuda_fail(e, "wavefront work list");
  }
  c.wave_nitems = (int)items.size();
  c.wave_par = 0;
  // persistent grid: every CTA that fits on the device at once (per phase:
  // the two step kernels differ in registers)
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, lat->device);
  for (int ph = 0; ph < 2 && e == cudaSuccess; ++ph) {
    int per_sm = 0;
    const void* fn = lat->storage == MLBM_STORE_F32 ? pick_wave<float>(ph, OUT_NONE)
                                                    : pick_wave<__half>(ph, OUT_NONE);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWaveThreads, 0);
    c.wave_grid[ph] = std::max(1, std::min(sms * std::max(1, per_sm), c.wave_nitems));
  }
  if (e != cudaSuccess) return cuda_fail(e, "wavefront occupancy");
  c.wave_built = true;
  return MLBM_OK;
}

}  // namespace

mlbm_status compact_set_wave_shape(mlbm_lattice* lat, int tile, int lookahead) {
  CompactState& c = lat->compact;
  c.wave_tile = tile;
  c.wave_lookahead = lookahead;
  c.wave_built = false;
  return MLBM_OK;
}

void compact_reset_wave(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  if (c.wave_ctl)
    cudaMemset(c.wave_ctl, 0, (2 + 2 * (size_t)lat->g.lz) * sizeof(unsigned));
  c.wave_par = 0;
}

template <typename T>
mlbm_status launch_compact_wave(mlbm_lattice* lat, const StepArgs& a,
                                bool write_u, bool write_rho) {
  CompactState& c = lat->compact;
  if (!c.wave_built)
    if (mlbm_status st = build_wave(lat)) return st;
  if (c.wave_nitems == 0) return MLBM_OK;
  const Phys& p = lat->phys;
  const bool inj = p.rho_inject_period != 0ull &&
                   (unsigned long long)a.step % p.rho_inject_period == 0ull;
  const int out = write_u ? (OUT_RHO | OUT_VEL) : (write_rho ? OUT_RHO : OUT_NONE);
  T* cpop = static_cast<T*>(c.cpop);
  uint32_t cs = (uint32_t)c.cs;
  int nf = (int)c.nfluid;
  const uint2* cinfo = c.cinfo;
  const uint2* wtab = c.wtab;
  float* rho = static_cast<float*>(lat->rho);
  float* psi = static_cast<float*>(lat->psi);
  float* vel = lat->vel;
  Geom g = lat->g;
  Phys pp = p;
  StepArgs aa = a;
  bool injv = inj;
  WaveArgs w;
  w.items = c.wave_items;
  w.need = c.wave_need;
  w.ticket = c.wave_ctl;
  w.done = c.wave_ctl + 2;
  w.err = lat->err;
  w.nitems = c.wave_nitems;
  w.lz = g.lz;
  w.par = c.wave_par;
  w.spin_limit = kWaveSpinLimit;
  void* args[] = {&cpop, &cs, &nf, &cinfo, &wtab, &rho, &psi, &vel, &g, &pp, &aa, &injv, &w};
  const cudaError_t e = cudaLaunchKernel(pick_wave<T>(lat->phase, out),
                                         dim3(c.wave_grid[lat->phase]),
                                         dim3(kWaveThreads),
                                         args, 0, lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wavefront time-step launch");
  c.wave_par ^= 1;
  return MLBM_OK;
}

template mlbm_status launch_compact_wave<float>(mlbm_lattice*, const StepArgs&, bool, bool);
template mlbm_status launch_compact_wave<__half>(mlbm_lattice*, const StepArgs&, bool, bool);

// ---- one-pass step (band.cuh) ---------------------------------------------------

namespace {

constexpr size_t kBandSmemMax = 227 * 1024;

// Bands of about `rows` rows along y and chunks of about `planes` planes
// along z; the tallest band's psi ring must fit shared memory.
BandShape band_shape(const Geom& g, int rows, int planes) {
  BandShape s;
  s.nb = std::max(1, g.ly / std::max(1, rows));
  s.nc = std::max(1, g.lz / std::max(1, planes));
  s.hmax = (g.ly + s.nb - 1) / s.nb;
  return s;
}

template <typename T, bool WR, bool WU>
const void* band_fn() {
  return reinterpret_cast<const void*>(&k_band<T, WR, WU>);
}

template <typename T>
const void* pick_band(bool wr, bool wu) {
  if (wu) return band_fn<T, true, true>();
  return wr ? band_fn<T, true, false>() : band_fn<T, false, false>();
}

// The dynamic shared-memory limit is an attribute of the kernel on each
// device: raise it (never lower it) to the largest size any lattice needs.
template <typename T>
mlbm_status band_smem_attr(int device, size_t smem) {
  static std::mutex mu;
  static size_t done[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device >= 0 && device < 64 && done[device] >= smem) return MLBM_OK;
  for (int v = 0; v < 3; ++v) {
    const cudaError_t e = cudaFuncSetAttribute(
        pick_band<T>(v >= 1, v == 2), cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "one-pass step attribute");
  }
  if (device >= 0 && device < 64) done[device] = smem;
  return MLBM_OK;
}

}  // namespace

bool compact_band_supported(const mlbm_lattice* lat, int rows) {
  if (!lat->compact.two_pass_ok || lat->slab) return false;
  const BandShape s = band_shape(lat->g, rows, 1);
  return band_smem_bytes(s.hmax, lat->g.lx) <= kBandSmemMax;
}

mlbm_status compact_set_band_shape(mlbm_lattice* lat, int rows, int planes) {
  if (!compact_band_supported(lat, rows))
    return set_error(MLBM_ERR_ARG,
                     "one-pass step: the bands' psi planes do not fit shared "
                     "memory (fewer rows per band, or the two-pass step)");
  lat->compact.band_rows = rows;
  lat->compact.band_planes = planes;
  return MLBM_OK;
}

template <typename T>
mlbm_status launch_compact_band(mlbm_lattice* lat, const StepArgs& a,
                                bool write_u, bool write_rho) {
  CompactState& c = lat->compact;
  if (lat->phase != 1)
    return set_error(MLBM_ERR_STATE, "one-pass step needs the AA phase-1 state");
  if (!c.cpop_alt) {
    const cudaError_t e =
        cudaMalloc(&c.cpop_alt, (size_t)c.cs * Q * pop_elem_bytes(lat->storage));
    if (e != cudaSuccess) {
      c.cpop_alt = nullptr;
      cudaGetLastError();
      return cuda_fail(e, "one-pass step buffer");
    }
  }
  const BandShape s = band_shape(lat->g, c.band_rows, c.band_planes);
  const size_t smem = band_smem_bytes(s.hmax, lat->g.lx);
  if (smem > kBandSmemMax)
    return set_error(MLBM_ERR_ARG, "one-pass step: band does not fit shared memory");
  if (mlbm_status st = band_smem_attr<T>(lat->device, smem)) return st;
  const bool inj = inject_now(lat, a);
  const T* A = static_cast<const T*>(c.cpop);
  T* B = static_cast<T*>(c.cpop_alt);
  const dim3 grid((unsigned)s.nb * (unsigned)s.nc);
  float* rho = static_cast<float*>(lat->rho);
  const uint32_t cs = (uint32_t)c.cs;
  if (write_u)
    k_band<T, true, true><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->g, lat->phys, a, inj, s);
  else if (write_rho)
    k_band<T, true, false><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->g, lat->phys, a, inj, s);
  else
    k_band<T, false, false><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->g, lat->phys, a, inj, s);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "one-pass step launch");
  std::swap(c.cpop, c.cpop_alt);
  return MLBM_OK;
}

template mlbm_status launch_compact_band<float>(mlbm_lattice*, const StepArgs&, bool, bool);
template mlbm_status launch_compact_band<__half>(mlbm_lattice*, const StepArgs&, bool, bool);

}  // namespace mlbm
