// compact.cu -- host side of the step kernels over the fluid-only layout
// (compact.cuh): tables built from the mask, layout changes, the two-pass
// launches (compact2.cuh) and the one-pass step (band.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "capi_internal.h"
#include "compact.cuh"
#include "band.cuh"
#include "compact2.cuh"

namespace mlbm {

namespace {

dim3 node_block() { return dim3(32, 4, 1); }
dim3 node_grid(const Geom& g) { return dim3(g.px / 32, (g.ly + 3) / 4, g.lz); }

CArgs args_of(const mlbm_lattice* lat) {
  const CompactState& c = lat->compact;
  CArgs a;
  a.mask = lat->mask;
  a.wbase = c.wbase;
  a.cs = c.cs;
  return a;
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
  c.row_start.assign((size_t)g.lz * g.ly + 1, 0);
  for (long long r = 0; r <= (long long)g.lz * g.ly; ++r)
    c.row_start[r] = h[r * g.wpr];
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
    cudaFree(c.cinfo);
    c.cpop = nullptr;
    c.cpop_alt = nullptr;
    c.cinfo = nullptr;
    c.cap = 0;
    e = cudaMalloc(&c.cpop, (size_t)c.cs * Q * pop_elem_bytes(lat->storage));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c.cinfo, (size_t)c.cs * sizeof(uint2));
    if (e != cudaSuccess) {
      cudaFree(c.cpop);
      c.cpop = nullptr;
      cudaGetLastError();
      return cuda_fail(e, "compact buffers");
    }
    c.cap = c.cs;
  }
  c.band_slot_rows = -1;  // stage sizes follow the tables
  c.built = true;
  return MLBM_OK;
}

template <typename T>
mlbm_status enter_t(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  const CArgs a = args_of(lat);
  // holes keep (0, 0): no fluid bit
  cudaError_t e = cudaMemsetAsync(c.cinfo, 0, c.cs * sizeof(uint2), lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "compact node table");
  k_cinfo<<<node_grid(lat->g), node_block(), 0, lat->stream>>>(lat->nbw, c.cinfo,
                                                                a, lat->g);
  // the layout change comes last: the first step's density pass, launched
  // with programmatic dependent launch, reads the node table before it
  // waits for the kernel before it (launch_overlapped)
  k_convert<T, true><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<T*>(lat->pop), static_cast<T*>(c.cpop), a, lat->g);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact entry launch");
  return MLBM_OK;
}

template <typename T>
mlbm_status to_dense_t(mlbm_lattice* lat) {
  const CArgs a = args_of(lat);
  k_convert<T, false><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<T*>(lat->pop), static_cast<T*>(lat->compact.cpop), a, lat->g);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact exit launch");
  return MLBM_OK;
}

}  // namespace

// Population offsets of the compact kernels are 32-bit (pair.cuh):
// Q * cs < 2^32 holds for every lattice of fewer than kC2MaxNodes nodes.
// (margin: up to one hole per plane and the rounding of cs to 64)
constexpr long long kC2MaxNodes = (1LL << 32) / Q - 4096;

bool compact_two_pass_supported(int lx, int ly, int lz, int storage) {
  return storage != MLBM_STORE_F64 && lx <= kC2MaxX && ly <= kC2MaxY &&
         lz <= kC2MaxZ && (long long)lx * ly * lz <= kC2MaxNodes;
}

mlbm_status compact_enter(mlbm_lattice* lat) {
  CompactState& c = lat->compact;
  if (c.active) return MLBM_OK;
  if (!c.two_pass_ok)
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
  cudaFree(c.cinfo);
  cudaFree(c.wbase);
  cudaFree(c.wtab);
  c = CompactState{};
}

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

// Launch a step kernel, with programmatic stream serialization when
// `overlap`: it may then begin while the kernel before it in the stream
// finishes, and waits for it at pdl_gate() (pair.cuh).  What a kernel reads
// before its gate must not be written by the kernel launched right before
// it, whose writes are visible only after the gate:
//   k_cdensity reads the node table (cinfo, wtab) before its gate; the
//     tables are written only in compact_enter, whose last kernel
//     (k_convert) does not write them;
//   k_cupdate also gathers populations before its gate; it is launched with
//     overlap only right after the density pass of the same step
//     (launch_compact_two_pass), which reads them only.  The slab pass API
//     (launch_compact_pass) may run halo moves between the passes, so it
//     launches without overlap.
template <typename... KArgs, typename... Args>
void launch_overlapped(bool overlap, void (*kernel)(KArgs...), unsigned grid,
                       cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kC2Threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = overlap ? 1 : 0;
  // a failed launch is reported by the caller's cudaGetLastError
  (void)cudaLaunchKernelEx(&cfg, kernel, args...);
}

unsigned c2_grid(long long kb, long long ke, long long per_thread) {
  const long long threads = (ke - kb + per_thread - 1) / per_thread;
  return (unsigned)((threads + kC2Threads - 1) / kC2Threads);
}

template <typename T, int PHASE>
void launch_c2_density(mlbm_lattice* lat, const StepArgs& a, bool wr, bool inj,
                       long long kb, long long ke, bool overlap) {
  const CompactState& c = lat->compact;
  const unsigned grid = c2_grid(kb, ke, c2_nodes_per_thread<PHASE>());
  if (grid == 0) return;
  const T* cpop = static_cast<const T*>(c.cpop);
  const uint32_t cs = (uint32_t)c.cs;
  float* rho = static_cast<float*>(lat->rho);
  float* psi = static_cast<float*>(lat->psi);
  auto kernel = wr ? k_cdensity<T, PHASE, true> : k_cdensity<T, PHASE, false>;
  launch_overlapped(overlap, kernel, grid, lat->stream, cpop, cs,
                    (const uint2*)c.cinfo, (const uint2*)c.wtab, (int)kb,
                    (int)ke, rho, psi, lat->g, lat->phys, a, inj);
}

template <typename T, int PHASE>
void launch_c2_update(mlbm_lattice* lat, const StepArgs& a, bool wu, bool inj,
                      long long kb, long long ke, bool overlap) {
  const unsigned grid = c2_grid(kb, ke, c2_update_nodes_per_thread());
  if (grid == 0) return;
  const CompactState& c = lat->compact;
  T* cpop = static_cast<T*>(c.cpop);
  const uint32_t cs = (uint32_t)c.cs;
  const float* psi = static_cast<const float*>(lat->psi);
  auto kernel = wu ? k_cupdate<T, PHASE, true> : k_cupdate<T, PHASE, false>;
  launch_overlapped(overlap, kernel, grid, lat->stream, cpop, cs,
                    (const uint2*)c.cinfo,
                    (const uint2*)c.wtab, (int)kb, (int)ke, psi, lat->vel,
                    lat->g, lat->phys, a, inj);
}

bool inject_now(const mlbm_lattice* lat, const StepArgs& a) {
  const Phys& p = lat->phys;
  return p.rho_inject_period != 0ull &&
         (unsigned long long)a.step % p.rho_inject_period == 0ull;
}
}  // namespace

namespace {
// Launches into a stream that is being captured into a CUDA graph are plain:
// the batched step's graphs with overlapped launches gave wrong states, so
// the overlap is used in ordinary stream order only.
bool stream_capturing(cudaStream_t stream) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &st) != cudaSuccess) {
    cudaGetLastError();  // a query refused during another capture: be plain
    return true;
  }
  return st != cudaStreamCaptureStatusNone;
}
}  // namespace

template <typename T>
mlbm_status launch_compact_two_pass(mlbm_lattice* lat, const StepArgs& a,
                                    bool write_u, bool write_rho) {
  const bool inj = inject_now(lat, a);
  long long kb, ke;
  own_range(lat, kb, ke);
  const bool overlap = !stream_capturing(lat->stream);
  if (lat->phase == 0) {
    launch_c2_density<T, 0>(lat, a, write_rho, inj, kb, ke, overlap);
    launch_c2_update<T, 0>(lat, a, write_u, inj, kb, ke, overlap);
  } else {
    launch_c2_density<T, 1>(lat, a, write_rho, inj, kb, ke, overlap);
    launch_c2_update<T, 1>(lat, a, write_u, inj, kb, ke, overlap);
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
    long long kb, ke;
    own_range(lat, kb, ke);
    if (lat->phase == 0) launch_c2_density<T, 0>(lat, a, write_rho, inj, kb, ke, false);
    else launch_c2_density<T, 1>(lat, a, write_rho, inj, kb, ke, false);
  } else {
    long long kb, ke;
    own_range(lat, kb, ke);
    if (lat->phase == 0) launch_c2_update<T, 0>(lat, a, write_u, inj, kb, ke, false);
    else launch_c2_update<T, 1>(lat, a, write_u, inj, kb, ke, false);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact pass launch");
  return MLBM_OK;
}

template mlbm_status launch_compact_pass<float>(mlbm_lattice*, const StepArgs&, int, bool, bool);
template mlbm_status launch_compact_pass<__half>(mlbm_lattice*, const StepArgs&, int, bool, bool);

// ---- one-pass step (band.cuh) ---------------------------------------------------

namespace {

constexpr size_t kBandSmemMax = 227 * 1024;

// Bands of about `rows` rows along y and chunks of about `planes` planes
// along z.
BandShape band_shape(const Geom& g, int rows, int planes) {
  BandShape s;
  s.nb = std::max(1, g.ly / std::max(1, rows));
  s.nc = std::max(1, g.lz / std::max(1, planes));
  s.hmax = (g.ly + s.nb - 1) / s.nb;
  s.slot = 0;
  return s;
}

// Compact slots one stage must hold for bands of shape s: the largest
// aligned extent of a band's rows y0 - 1 .. y1 over all bands and planes
// (band_ranges), plus one alignment unit so a pair load at a range's end
// stays inside the stage.
int band_slot(const mlbm_lattice* lat, const BandShape& s, int align) {
  const CompactState& c = lat->compact;
  const Geom& g = lat->g;
  long long mx = 0;
  for (int b = 0; b < s.nb; ++b) {
    const int y0 = (int)((long long)b * g.ly / s.nb);
    const int y1 = (int)((long long)(b + 1) * g.ly / s.nb);
    int ra[2], rb[2];
    const int n = band_row_ranges(g.ly, y0, y1, ra, rb);
    for (int z = 0; z < g.lz; ++z) {
      long long tot = 0;
      for (int q = 0; q < n; ++q) {
        const long long kf = c.row_start[(size_t)z * g.ly + ra[q]];
        const long long ke = c.row_start[(size_t)z * g.ly + rb[q]];
        tot += (ke + align - 1) / align * align - kf / align * align;
      }
      mx = std::max(mx, tot);
    }
  }
  return (int)(mx + align);
}

// The band shape a launch uses: the requested rows, lowered until the psi
// ring and the stages fit shared memory (0 bands: nothing fits).
template <typename T>
BandShape fit_band_shape(mlbm_lattice* lat, int rows, int planes) {
  CompactState& c = lat->compact;
  for (int r = std::max(1, rows); r >= 1; --r) {
    BandShape s = band_shape(lat->g, r, planes);
    if (c.band_slot_rows == r && c.band_slot_nb == s.nb &&
        c.band_slot_storage == lat->storage) {
      s.slot = c.band_slot;
    } else {
      s.slot = band_slot(lat, s, band_align<T>());
      c.band_slot = s.slot;
      c.band_slot_rows = r;
      c.band_slot_nb = s.nb;
      c.band_slot_storage = lat->storage;
    }
    if (band_smem_bytes<T>(s.hmax, lat->g.lx, s.slot) <= kBandSmemMax) return s;
  }
  BandShape none = band_shape(lat->g, 1, planes);
  none.nb = 0;
  return none;
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

bool compact_band_supported(const mlbm_lattice* lat) {
  return lat->compact.two_pass_ok && !lat->slab;
}

bool compact_band_fits(mlbm_lattice* lat) {
  if (!lat->compact.built) return false;
  const BandShape s =
      lat->storage == MLBM_STORE_F16
          ? fit_band_shape<__half>(lat, lat->compact.band_rows, lat->compact.band_planes)
          : fit_band_shape<float>(lat, lat->compact.band_rows, lat->compact.band_planes);
  return s.nb > 0;
}

mlbm_status compact_set_band_shape(mlbm_lattice* lat, int rows, int planes) {
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
  const BandShape s = fit_band_shape<T>(lat, c.band_rows, c.band_planes);
  if (s.nb == 0)
    return set_error(MLBM_ERR_ARG, "one-pass step: a band does not fit shared memory");
  const size_t smem = band_smem_bytes<T>(s.hmax, lat->g.lx, s.slot);
  if (mlbm_status st = band_smem_attr<T>(lat->device, smem)) return st;
  const bool inj = inject_now(lat, a);
  const bool stall = lat->stall_test;
  lat->stall_test = false;
  const T* A = static_cast<const T*>(c.cpop);
  T* B = static_cast<T*>(c.cpop_alt);
  const dim3 grid((unsigned)s.nb * (unsigned)s.nc);
  float* rho = static_cast<float*>(lat->rho);
  const uint32_t cs = (uint32_t)c.cs;
  if (write_u)
    k_band<T, true, true><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->err, lat->g, lat->phys,
        a, inj, s, lat->wait_ns, stall);
  else if (write_rho)
    k_band<T, true, false><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->err, lat->g, lat->phys,
        a, inj, s, lat->wait_ns, stall);
  else
    k_band<T, false, false><<<grid, kBandThreads, smem, lat->stream>>>(
        A, B, cs, c.cinfo, c.wtab, rho, lat->vel, lat->err, lat->g, lat->phys,
        a, inj, s, lat->wait_ns, stall);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "one-pass step launch");
  std::swap(c.cpop, c.cpop_alt);
  return MLBM_OK;
}

template mlbm_status launch_compact_band<float>(mlbm_lattice*, const StepArgs&, bool, bool);
template mlbm_status launch_compact_band<__half>(mlbm_lattice*, const StepArgs&, bool, bool);

}  // namespace mlbm
