// capi.cu -- implementation of the C ABI in include/mlbm.h.
//
// Owns the device memory of each lattice and issues the kernels of
// kernels.cuh / io_kernels.cuh on the lattice's stream.  Host-side errors are
// returned as mlbm_status with a message kept per host thread; nothing here
// exits or falls back to the CPU.
#include <cuda_runtime.h>
#include <type_traits>

#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "../../include/mlbm.h"
#include "capi_internal.h"
#include "io_kernels.cuh"
#include "kernels.cuh"
#include "update_tma.cuh"

using namespace mlbm;

namespace {

thread_local std::string g_last_error;

mlbm_status fail(mlbm_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

}  // namespace

namespace mlbm {

mlbm_status set_error(mlbm_status st, const char* msg) {
  g_last_error = msg;
  return st;
}

mlbm_status cuda_fail(cudaError_t e, const char* where) {
  if (e == cudaErrorMemoryAllocation)
    return fail(MLBM_ERR_NOMEM, "%s: %s", where, cudaGetErrorString(e));
  return fail(MLBM_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

size_t pop_elem_bytes(int storage) {
  return storage == MLBM_STORE_F16 ? 2 : (storage == MLBM_STORE_F64 ? 8 : 4);
}
size_t real_bytes(int storage) { return storage == MLBM_STORE_F64 ? 8 : 4; }

Geom make_geom(int lx, int ly, int lz) {
  Geom g;
  g.lx = lx;
  g.ly = ly;
  g.lz = lz;
  g.px = (lx + 31) / 32 * 32;
  g.wpr = g.px / 32;
  g.plane = (long long)lz * ly * g.px;
  g.pxg = g.px + 8;
  return g;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
mlbm_status setup_update(mlbm_lattice* lat, int rows, int planes) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                              void*, const cuuint64_t*, const cuuint64_t*,
                              const cuuint32_t*, const cuuint32_t*,
                              CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault,
                                &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return set_error(MLBM_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    }
    encode = reinterpret_cast<Encode>(fn);
  }
  const Geom& g = lat->g;
  ZMarch& zm = lat->zm;
  zm.By = std::max(1, std::min(rows, 8));
  zm.Dz = std::max(1, planes);
  zm.ntx = g.px / 32;
  zm.nty = (g.ly + zm.By - 1) / zm.By;
  zm.nzc = (g.lz + zm.Dz - 1) / zm.Dz;
  const bool f64 = lat->storage == MLBM_STORE_F64;
  const size_t esz = f64 ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)g.pxg, (cuuint64_t)(g.ly + 2),
                        (cuuint64_t)(g.lz + 2)};
  cuuint64_t strides[2] = {(cuuint64_t)g.pxg * esz,
                           (cuuint64_t)g.pxg * (g.ly + 2) * esz};
  cuuint32_t box[3] = {(cuuint32_t)kBoxX, (cuuint32_t)(zm.By + 2), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(
      &lat->psi_map,
      f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
      lat->psi, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(MLBM_ERR_CUDA, "psi tensor map could not be encoded");
  return MLBM_OK;
}

}  // namespace mlbm

#define CUDA_TRY(expr, where)                           \
  do {                                                  \
    cudaError_t _e = (expr);                            \
    if (_e != cudaSuccess) return mlbm::cuda_fail(_e, where); \
  } while (0)

namespace {

dim3 node_block() { return dim3(32, 4, 1); }
dim3 node_grid(const Geom& g) {
  return dim3(g.px / 32, (g.ly + 3) / 4, g.lz);
}

Phys to_phys(const mlbm_params& p) {
  Phys q;
  q.tau = p.tau;
  q.G = p.G;
  q.T_Tc = p.T_Tc;
  q.rhol_spinodal = p.rhol_spinodal;
  q.rhog_spinodal = p.rhog_spinodal;
  q.rhos = p.rhos;
  q.rho_increment = p.rho_increment;
  q.inject_position = p.inject_position;
  q.carn_star = p.carn_star;
  q.rho_inject_period = p.rho_inject_period;
  q.inlet_width = p.inlet_width;
  q.outlet_width = p.outlet_width;
  q.rho_inlet = p.rho_inlet;
  q.rho_outlet = p.rho_outlet;
  q.rho_shift = p.rho_shift;
  q.omega = (float)(1.0 / (double)p.tau);
  return q;
}

mlbm_status check_lat(const mlbm_lattice* lat) {
  if (!lat) return fail(MLBM_ERR_ARG, "null lattice handle");
  return MLBM_OK;
}

mlbm_status activate(const mlbm_lattice* lat) {
  CUDA_TRY(cudaSetDevice(lat->device), "cudaSetDevice");
  return MLBM_OK;
}

template <typename T, int PHASE>
void launch_density(mlbm_lattice* lat, const StepArgs& a, bool write_rho) {
  using R = typename Pop<T>::Real;
  const T* pop = static_cast<const T*>(lat->pop);
  R* rho = static_cast<R*>(lat->rho);
  R* psi = static_cast<R*>(lat->psi);
  if (write_rho)
    k_density<T, PHASE, true><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        pop, lat->nbw, rho, psi, lat->g, lat->phys, a);
  else
    k_density<T, PHASE, false><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        pop, lat->nbw, rho, psi, lat->g, lat->phys, a);
}

template <typename T, int PHASE, bool WU>
void launch_update(mlbm_lattice* lat, const StepArgs& a) {
  using R = typename Pop<T>::Real;
  const ZMarch& zm = lat->zm;
  const size_t smem = update_smem_bytes(zm.By, sizeof(R));
  k_update_zm<T, PHASE, WU>
      <<<zm.ntx * zm.nty * zm.nzc, 32 * zm.By, smem, lat->stream>>>(
          static_cast<T*>(lat->pop), lat->nbw, lat->vel, lat->err, lat->g,
          lat->phys, a, zm, lat->psi_map);
}

template <typename T>
mlbm_status launch_two_pass(mlbm_lattice* lat, const StepArgs& a, bool wu,
                            bool write_rho) {
  if (lat->phase == 0) {
    launch_density<T, 0>(lat, a, write_rho);
    if (wu) launch_update<T, 0, true>(lat, a);
    else launch_update<T, 0, false>(lat, a);
  } else {
    launch_density<T, 1>(lat, a, write_rho);
    if (wu) launch_update<T, 1, true>(lat, a);
    else launch_update<T, 1, false>(lat, a);
  }
  CUDA_TRY(cudaGetLastError(), "time-step launch");
  return MLBM_OK;
}

// One lattice step per launch (two launches for the two-pass kernels, which
// AUTO selects).  rho is written on the last step of each mlbm_iterate call
// (the field the caller can read afterwards).
// The step kernel a lattice runs: AUTO is the compact two-pass step where it
// supports the lattice (FP32 / FP16 storage), else the dense two-pass step.
int effective_kernel(const mlbm_lattice* lat) {
  if (lat->step_kernel != MLBM_KERNEL_AUTO) return lat->step_kernel;
  return lat->compact.two_pass_ok ? MLBM_KERNEL_COMPACT : MLBM_KERNEL_TWO_PASS;
}

template <typename T>
mlbm_status launch_steps(mlbm_lattice* lat, int64_t step0, int32_t nsteps,
                         int32_t reverse, uint32_t inject_type,
                         uint32_t flags) {
  const int kind = effective_kernel(lat);
  bool compact = false, band = false;
  if constexpr (!std::is_same<T, double>::value) {
    compact = kind == MLBM_KERNEL_COMPACT || kind == MLBM_KERNEL_BAND;
    band = kind == MLBM_KERNEL_BAND;
  }
  if ((flags & MLBM_ITER_WRITE_VELOCITY) && !lat->vel) {
    // the velocity field is allocated on first request
    CUDA_TRY(cudaMalloc((void**)&lat->vel, (size_t)lat->g.plane * 3 * sizeof(float)),
             "velocity allocation");
    // solid nodes are never written: they read zero velocity
    CUDA_TRY(cudaMemsetAsync(lat->vel, 0, (size_t)lat->g.plane * 3 * sizeof(float),
                             lat->stream),
             "velocity clear");
  }
  if (compact) {
    if (mlbm_status st = compact_enter(lat)) return st;
    // bands that do not fit shared memory: compact two-pass steps
    if (band && !compact_band_fits(lat)) band = false;
  } else {
    if (mlbm_status st = compact_leave(lat)) return st;
  }
  for (int32_t s = 0; s < nsteps; ++s) {
    StepArgs a{(long long)(step0 + s), reverse, inject_type};
    const bool last = s == nsteps - 1;
    const bool wu = (flags & MLBM_ITER_WRITE_VELOCITY) && last;
    mlbm_status st;
    // the one-pass step starts and ends in AA phase 1; from phase 0 one
    // two-pass step gets there
    const bool one_pass = band && lat->phase == 1;
    if constexpr (!std::is_same<T, double>::value) {
      if (one_pass) st = launch_compact_band<T>(lat, a, wu, last);
      else if (compact) st = launch_compact_two_pass<T>(lat, a, wu, last);
      else st = launch_two_pass<T>(lat, a, wu, last);
    } else {
      st = launch_two_pass<T>(lat, a, wu, last);
    }
    if (st) return st;
    if (!one_pass) lat->phase ^= 1;
    if (wu) lat->vel_valid = true;
  }
  return MLBM_OK;
}

template <typename T>
mlbm_status launch_init(mlbm_lattice* lat) {
  using R = typename Pop<T>::Real;
  k_build_nbr<<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      lat->mask, lat->nbw, lat->g, lat->phys);
  k_init<T><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<T*>(lat->pop), lat->mask, lat->rho_init,
      static_cast<R*>(lat->rho), static_cast<R*>(lat->psi), lat->g, lat->phys);
  CUDA_TRY(cudaGetLastError(), "init launch");
  return MLBM_OK;
}

template <typename T, typename O>
void launch_pop_out(mlbm_lattice* lat, O* out) {
  k_pop_to_ref<T, O><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<const T*>(lat->pop), lat->mask, out, lat->g, lat->phys,
      lat->phase);
}

template <typename R, typename O>
void launch_scalar_out(mlbm_lattice* lat, int field, O* out) {
  k_scalar_to_ref<R, O><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
      static_cast<const R*>(lat->rho), lat->mask, out, lat->g, lat->phys,
      field);
}

template <typename O>
mlbm_status field_out(mlbm_lattice* lat, int32_t field, O* dev_out) {
  switch (field) {
    case MLBM_FIELD_RHO:
    case MLBM_FIELD_PRESSURE:
    case MLBM_FIELD_PSI:
      if (lat->storage == MLBM_STORE_F64)
        launch_scalar_out<double, O>(lat, field, dev_out);
      else
        launch_scalar_out<float, O>(lat, field, dev_out);
      break;
    case MLBM_FIELD_VELOCITY:
      if (!lat->vel_valid)
        return fail(MLBM_ERR_STATE,
                    "velocity not written: iterate with "
                    "MLBM_ITER_WRITE_VELOCITY first");
      k_vel_to_ref<O><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
          lat->vel, dev_out, lat->g);
      break;
    case MLBM_FIELD_POPULATIONS:
      if (mlbm_status st = compact_sync_dense(lat)) return st;
      if (lat->storage == MLBM_STORE_F32)
        launch_pop_out<float, O>(lat, dev_out);
      else if (lat->storage == MLBM_STORE_F16)
        launch_pop_out<__half, O>(lat, dev_out);
      else
        launch_pop_out<double, O>(lat, dev_out);
      break;
    default:
      return fail(MLBM_ERR_ARG, "unknown field %d", field);
  }
  CUDA_TRY(cudaGetLastError(), "field download launch");
  return MLBM_OK;
}

size_t field_components(int32_t field) {
  return field == MLBM_FIELD_VELOCITY ? 3
         : field == MLBM_FIELD_POPULATIONS ? Q
                                           : 1;
}

// After a stream synchronisation: report (and clear) a wait timeout raised by
// a step kernel.  The interrupted step left the lattice inconsistent.
mlbm_status check_device_error(mlbm_lattice* lat) {
  int h = 0;
  CUDA_TRY(cudaMemcpy(&h, lat->err, sizeof(int), cudaMemcpyDeviceToHost),
           "error flag read");
  if (!h) return MLBM_OK;
  cudaMemset(lat->err, 0, sizeof(int));
  lat->initialized = false;
  return fail(MLBM_ERR_TIMEOUT,
              "a bounded wait of the time step ran out; the lattice must be "
              "initialised again");
}

mlbm_status ensure_staging(mlbm_lattice* lat, size_t bytes) {
  if (lat->staging_bytes >= bytes) return MLBM_OK;
  if (lat->staging) cudaFree(lat->staging);
  lat->staging = nullptr;
  lat->staging_bytes = 0;
  CUDA_TRY(cudaMalloc(&lat->staging, bytes), "staging allocation");
  lat->staging_bytes = bytes;
  return MLBM_OK;
}

}  // namespace

// ============================================================================
extern "C" {

int32_t mlbm_abi_version(void) { return MLBM_ABI_VERSION; }

const char* mlbm_status_string(int32_t s) {
  switch (s) {
    case MLBM_OK: return "ok";
    case MLBM_ERR_ARG: return "invalid argument";
    case MLBM_ERR_CUDA: return "CUDA error";
    case MLBM_ERR_NOMEM: return "out of device memory";
    case MLBM_ERR_STATE: return "call out of order";
    case MLBM_ERR_TIMEOUT: return "device wait timed out";
    case MLBM_ERR_IO: return "I/O error";
    case MLBM_ERR_PARSE: return "parse error";
  }
  return "unknown status";
}

const char* mlbm_last_error(void) { return g_last_error.c_str(); }

void mlbm_d3q19(int32_t* e, float* w) {
  for (int i = 0; i < Q; ++i) {
    if (e) {
      e[3 * i] = ex(i);
      e[3 * i + 1] = ey(i);
      e[3 * i + 2] = ez(i);
    }
    if (w) w[i] = weight<float>(i);
  }
}

uint64_t mlbm_lattice_bytes(int32_t lx, int32_t ly, int32_t lz,
                            int32_t storage) {
  if (lx <= 0 || ly <= 0 || lz <= 0) return 0;
  const Geom g = make_geom(lx, ly, lz);
  const uint64_t np = (uint64_t)g.plane;
  return np * Q * pop_elem_bytes(storage)     // populations
         + np * real_bytes(storage)           // rho
         + (uint64_t)psi_elems(g) * real_bytes(storage)  // psi with ghosts
         + np * 4                             // initial density
         + (uint64_t)g.lz * g.ly * g.wpr * 4  // mask
         + np * 4;                            // neighbour words
  // (the velocity field, 12 bytes per node, is allocated on first request)
}

mlbm_status mlbm_lattice_create(int32_t lx, int32_t ly, int32_t lz,
                                int32_t storage, int32_t device,
                                mlbm_lattice** out) {
  if (!out) return fail(MLBM_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (lx < 1 || ly < 1 || lz < 1 || lz > 65535 || ly > (1 << 24) ||
      lx > (1 << 24))
    return fail(MLBM_ERR_ARG, "invalid lattice size %d x %d x %d", lx, ly, lz);
  if (make_geom(lx, ly, lz).plane >= (1LL << 31))
    return fail(MLBM_ERR_ARG, "lattice too large (more than 2^31 padded nodes)");
  if (storage < MLBM_STORE_F32 || storage > MLBM_STORE_F64)
    return fail(MLBM_ERR_ARG, "invalid storage %d", storage);
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev)
    return fail(MLBM_ERR_CUDA, "device %d not available (%d devices)", device,
                ndev);
  mlbm::DeviceGuard restore_device;
  CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
  mlbm_lattice* lat = new (std::nothrow) mlbm_lattice();
  if (!lat) return fail(MLBM_ERR_NOMEM, "host allocation failed");
  lat->device = device;
  lat->storage = storage;
  lat->g = make_geom(lx, ly, lz);
  lat->compact.two_pass_ok = compact_two_pass_supported(lx, ly, lz, storage);
  const size_t np = (size_t)lat->g.plane;
  const size_t mask_words = (size_t)lz * ly * lat->g.wpr;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  alloc(&lat->pop, np * Q * pop_elem_bytes(storage));
  alloc(&lat->rho, np * real_bytes(storage));
  alloc(&lat->psi, (size_t)psi_elems(lat->g) * real_bytes(storage));
  alloc((void**)&lat->rho_init, np * sizeof(float));
  alloc((void**)&lat->mask, mask_words * sizeof(uint32_t));
  alloc((void**)&lat->nbw, np * sizeof(uint32_t));
  alloc((void**)&lat->err, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemset(lat->psi, 0, (size_t)psi_elems(lat->g) * real_bytes(storage));
  if (e == cudaSuccess) e = cudaMemset(lat->err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(lat->mask, 0, mask_words * 4);
  if (e == cudaSuccess) e = cudaMemset(lat->rho_init, 0, np * sizeof(float));
  if (e != cudaSuccess) {
    mlbm_lattice_destroy(lat);
    cudaGetLastError();
    return cuda_fail(e, "lattice allocation");
  }
  if (mlbm_status st = setup_update(lat, 4, 16)) {
    mlbm_lattice_destroy(lat);
    return st;
  }
  *out = lat;
  return MLBM_OK;
}

mlbm_status mlbm_lattice_destroy(mlbm_lattice* lat) {
  if (!lat) return MLBM_OK;
  mlbm::DeviceGuard restore_device;
  cudaSetDevice(lat->device);
  if (lat->stream_owned_sync) cudaStreamSynchronize(lat->stream);
  cudaFree(lat->pop);
  cudaFree(lat->rho);
  cudaFree(lat->psi);
  cudaFree(lat->rho_init);
  cudaFree(lat->mask);
  cudaFree(lat->vel);
  cudaFree(lat->nbw);
  cudaFree(lat->staging);
  cudaFree(lat->stats_scratch);
  cudaFree(lat->err);
  compact_free(lat);
  delete lat;
  return MLBM_OK;
}

mlbm_status mlbm_set_stream(mlbm_lattice* lat, void* stream) {
  if (mlbm_status st = check_lat(lat)) return st;
  lat->stream = static_cast<cudaStream_t>(stream);
  return MLBM_OK;
}

mlbm_status mlbm_set_params(mlbm_lattice* lat, const mlbm_params* p) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!p) return fail(MLBM_ERR_ARG, "null params");
  if (!(p->tau > 0.f)) return fail(MLBM_ERR_ARG, "tau must be > 0 (got %g)", p->tau);
  if (p->inlet_width < 0 || p->outlet_width < 0 ||
      p->inlet_width + p->outlet_width > lat->g.lx)
    return fail(MLBM_ERR_ARG, "invalid drainage slab widths %d, %d",
                p->inlet_width, p->outlet_width);
  if (p->carn_star && p->G == 0.f)
    return fail(MLBM_ERR_ARG, "Carnahan-Starling psi needs G != 0");
  lat->params = *p;
  lat->phys = to_phys(*p);
  lat->has_params = true;
  return MLBM_OK;
}

static mlbm_status upload_mask_impl(mlbm_lattice* lat, const uint8_t* src,
                                    cudaMemcpyKind kind) {
  const Geom& g = lat->g;
  const size_t n = (size_t)g.lx * g.ly * g.lz;
  if (mlbm_status st = ensure_staging(lat, n)) return st;
  CUDA_TRY(cudaMemcpyAsync(lat->staging, src, n, kind, lat->stream),
           "mask upload copy");
  k_pack_mask<<<node_grid(g), node_block(), 0, lat->stream>>>(
      static_cast<const uint8_t*>(lat->staging), lat->mask, g);
  CUDA_TRY(cudaGetLastError(), "mask pack launch");
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "mask upload");
  compact_invalidate(lat);
  lat->has_mask = true;
  lat->initialized = false;
  return MLBM_OK;
}

static mlbm_status upload_rho_impl(mlbm_lattice* lat, const float* src,
                                   cudaMemcpyKind kind) {
  const Geom& g = lat->g;
  const size_t n = (size_t)g.lx * g.ly * g.lz;
  if (mlbm_status st = ensure_staging(lat, n * sizeof(float))) return st;
  CUDA_TRY(cudaMemcpyAsync(lat->staging, src, n * sizeof(float), kind,
                           lat->stream),
           "rho upload copy");
  k_rho_from_ref<<<node_grid(g), node_block(), 0, lat->stream>>>(
      static_cast<const float*>(lat->staging), lat->rho_init, g);
  CUDA_TRY(cudaGetLastError(), "rho transpose launch");
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "rho upload");
  lat->has_rho = true;
  lat->initialized = false;
  return MLBM_OK;
}

mlbm_status mlbm_upload_fluid_mask(mlbm_lattice* lat, const uint8_t* f) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!f) return fail(MLBM_ERR_ARG, "null mask");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  return upload_mask_impl(lat, f, cudaMemcpyDefault);
}
mlbm_status mlbm_upload_fluid_mask_device(mlbm_lattice* lat, const uint8_t* f) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!f) return fail(MLBM_ERR_ARG, "null mask");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  return upload_mask_impl(lat, f, cudaMemcpyDeviceToDevice);
}
mlbm_status mlbm_upload_rho(mlbm_lattice* lat, const float* r) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!r) return fail(MLBM_ERR_ARG, "null rho");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  return upload_rho_impl(lat, r, cudaMemcpyDefault);
}
mlbm_status mlbm_upload_rho_device(mlbm_lattice* lat, const float* r) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!r) return fail(MLBM_ERR_ARG, "null rho");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  return upload_rho_impl(lat, r, cudaMemcpyDeviceToDevice);
}

mlbm_status mlbm_initialize(mlbm_lattice* lat) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!lat->has_params || !lat->has_mask || !lat->has_rho)
    return fail(MLBM_ERR_STATE,
                "initialize needs params, fluid mask and rho first");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  mlbm_status st;
  switch (lat->storage) {
    case MLBM_STORE_F32: st = launch_init<float>(lat); break;
    case MLBM_STORE_F16: st = launch_init<__half>(lat); break;
    default: st = launch_init<double>(lat); break;
  }
  if (st) return st;
  lat->compact.active = false;  // the initial state is written densely
  lat->phase = 0;
  lat->initialized = true;
  lat->vel_valid = false;
  return MLBM_OK;
}

mlbm_status mlbm_iterate(mlbm_lattice* lat, int64_t step0, int32_t nsteps,
                         int32_t reverse, uint32_t inject_type,
                         uint32_t flags) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!lat->initialized)
    return fail(MLBM_ERR_STATE, "iterate before initialize");
  if (nsteps < 0) return fail(MLBM_ERR_ARG, "negative step count");
  if (lat->slab)
    return fail(MLBM_ERR_STATE,
                "iterate on a slab lattice: step it with mlbm_step_pass and "
                "exchange its halos between the passes");
  if (nsteps == 0) return MLBM_OK;
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  switch (lat->storage) {
    case MLBM_STORE_F32:
      return launch_steps<float>(lat, step0, nsteps, reverse, inject_type, flags);
    case MLBM_STORE_F16:
      return launch_steps<__half>(lat, step0, nsteps, reverse, inject_type, flags);
    default:
      return launch_steps<double>(lat, step0, nsteps, reverse, inject_type, flags);
  }
}

mlbm_status mlbm_download_field_device(mlbm_lattice* lat, int32_t field,
                                       int32_t dtype, void* dev_out) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!dev_out) return fail(MLBM_ERR_ARG, "null output");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  if (field == MLBM_FIELD_FLUID) {
    if (dtype != MLBM_DTYPE_U8)
      return fail(MLBM_ERR_ARG, "the fluid mask downloads as MLBM_DTYPE_U8");
    k_fluid_to_ref<<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        lat->mask, static_cast<uint8_t*>(dev_out), lat->g);
    CUDA_TRY(cudaGetLastError(), "mask download launch");
    return MLBM_OK;
  }
  if (!lat->initialized)
    return fail(MLBM_ERR_STATE, "field download before initialize");
  if (dtype == MLBM_DTYPE_F32)
    return field_out<float>(lat, field, static_cast<float*>(dev_out));
  if (dtype == MLBM_DTYPE_F64)
    return field_out<double>(lat, field, static_cast<double*>(dev_out));
  return fail(MLBM_ERR_ARG, "invalid dtype %d for field %d", dtype, field);
}

mlbm_status mlbm_download_field(mlbm_lattice* lat, int32_t field,
                                int32_t dtype, void* host_out) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!host_out) return fail(MLBM_ERR_ARG, "null output");
  const Geom& g = lat->g;
  const size_t esz = dtype == MLBM_DTYPE_F64 ? 8 : (dtype == MLBM_DTYPE_U8 ? 1 : 4);
  const size_t bytes = (size_t)g.lx * g.ly * g.lz * field_components(field) * esz;
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  if (mlbm_status st = ensure_staging(lat, bytes)) return st;
  if (mlbm_status st = mlbm_download_field_device(lat, field, dtype, lat->staging))
    return st;
  // cudaMemcpyDefault: host_out may be pageable, pinned or managed memory
  CUDA_TRY(cudaMemcpyAsync(host_out, lat->staging, bytes, cudaMemcpyDefault,
                           lat->stream),
           "field download copy");
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "field download");
  return check_device_error(lat);
}

}  // extern "C"

namespace {

// Enqueue the phase statistics reduction and the copy of its ST_COUNT + 1
// doubles (the last one the device error flag) to host memory `h`; `full`
// false: the bulk columns only (stat_node<R, false>).
mlbm_status stats_enqueue(mlbm_lattice* lat, double* h, bool full) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!h) return fail(MLBM_ERR_ARG, "null output");
  if (!lat->initialized) return fail(MLBM_ERR_STATE, "stats before initialize");
  if (lat->slab)
    return fail(MLBM_ERR_STATE,
                "phase statistics of a slab would count its halo planes: "
                "gather the slabs' own planes first");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  // a lattice held in the fluid-only layout is walked through its node
  // table (no lanes idle on solid nodes); otherwise the dense grid
  const CompactState& c = lat->compact;
  const bool fluid_list = c.active && c.cinfo && lat->storage != MLBM_STORE_F64;
  const dim3 grid(lat->g.px / 32, (lat->g.ly + 7) / 8,
                  (lat->g.lz + kStatZ - 1) / kStatZ);
  // The fluid-list form runs one wave of resident blocks over even spans of
  // the node table (spans of whole 256-slot rounds; one block at least: the
  // last block to finish writes the results).
  long long nblocks = (long long)grid.x * grid.y * grid.z, span = 0;
  if (fluid_list) {
    // Both forms use the full form's wave: the spans, and with them the
    // order of every sum, are then the same, so the bulk columns come out
    // bit-identical.
    if (lat->stats_wave <= 0) {
      int per_sm = 0, nsm = 0;
      CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &per_sm, k_stats_fluid<float, true>, kStatThreads, 0),
               "stats occupancy");
      CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount,
                                      lat->device),
               "stats occupancy");
      lat->stats_wave = std::max(1, per_sm * nsm);
    }
    const long long rounds =
        std::max(1LL, (c.nfluid + kStatThreads - 1) / kStatThreads);
    nblocks = std::min<long long>(lat->stats_wave, rounds);
    span = (rounds + nblocks - 1) / nblocks * kStatThreads;
    nblocks = std::max(1LL, (c.nfluid + span - 1) / span);
  }
  // slot 0: the arrival counter; the block records; the results
  const size_t need = (1 + (size_t)nblocks * ST_COUNT + ST_COUNT + 1) * sizeof(double);
  if (lat->stats_scratch_bytes < need) {
    // a larger area: earlier calls may still be reading the old one
    CUDA_TRY(cudaStreamSynchronize(lat->stream), "stats");
    cudaFree(lat->stats_scratch);
    lat->stats_scratch = nullptr;
    lat->stats_scratch_bytes = 0;
    CUDA_TRY(cudaMalloc((void**)&lat->stats_scratch, need), "stats scratch");
    CUDA_TRY(cudaMemsetAsync(lat->stats_scratch, 0, sizeof(double), lat->stream),
             "stats counter");
    lat->stats_scratch_bytes = need;
  }
  StatScratch sc;
  sc.counter = reinterpret_cast<unsigned*>(lat->stats_scratch);
  sc.records = lat->stats_scratch + 1;
  sc.out = sc.records + (size_t)nblocks * ST_COUNT;
  double* fin = sc.out;
  if (fluid_list) {
    auto kernel = full ? k_stats_fluid<float, true> : k_stats_fluid<float, false>;
    kernel<<<(unsigned)nblocks, kStatThreads, 0, lat->stream>>>(
        static_cast<const float*>(lat->rho), c.cinfo, c.nfluid, span, lat->g,
        lat->phys, sc, lat->err);
  } else if (lat->storage == MLBM_STORE_F64) {
    auto kernel = full ? k_stats_partial<double, true> : k_stats_partial<double, false>;
    kernel<<<grid, dim3(32, 8), 0, lat->stream>>>(
        static_cast<const double*>(lat->rho), lat->nbw, lat->g, lat->phys, sc,
        lat->err);
  } else {
    auto kernel = full ? k_stats_partial<float, true> : k_stats_partial<float, false>;
    kernel<<<grid, dim3(32, 8), 0, lat->stream>>>(
        static_cast<const float*>(lat->rho), lat->nbw, lat->g, lat->phys, sc,
        lat->err);
  }
  CUDA_TRY(cudaGetLastError(), "stats launch");
  CUDA_TRY(cudaMemcpyAsync(h, fin, (ST_COUNT + 1) * sizeof(double),
                           cudaMemcpyDeviceToHost, lat->stream),
           "stats copy");
  return MLBM_OK;
}

mlbm_status stats_convert(mlbm_lattice* lat, const double* h, mlbm_stats* out) {
  // the error flag came back with the statistics
  if (h[ST_COUNT] != 0.0)
    if (mlbm_status st = check_device_error(lat)) return st;
  std::memset(out, 0, sizeof *out);
  out->n_fluid = (int64_t)h[ST_NF];
  out->n_liquid = (int64_t)h[ST_NL];
  out->n_vapour = (int64_t)h[ST_NV];
  out->n_liquid_solid_boundary = (int64_t)h[ST_NLS];
  out->n_liquid_vapour_boundary = (int64_t)h[ST_NLV];
  out->mass = h[ST_MASS];
  out->sum_p_liquid = h[ST_PL];
  out->sum_p_vapour = h[ST_PV];
  out->sum_rho_liquid = h[ST_RL];
  out->sum_rho_vapour = h[ST_RV];
  out->saturation = out->n_fluid ? h[ST_NL] / h[ST_NF] : 0.0;
  if (out->n_liquid) {
    out->avg_p_liquid = h[ST_PL] / h[ST_NL];
    out->avg_rho_liquid = h[ST_RL] / h[ST_NL];
    out->ratio_liquid_solid_boundary = h[ST_NLS] / h[ST_NL];
    out->ratio_liquid_vapour_boundary = h[ST_NLV] / h[ST_NL];
  }
  if (out->n_vapour) {
    out->avg_p_vapour = h[ST_PV] / h[ST_NV];
    out->avg_rho_vapour = h[ST_RV] / h[ST_NV];
  }
  out->suction = out->avg_p_vapour - out->avg_p_liquid;
  out->min_rho = h[ST_MINR];
  out->max_rho = h[ST_MAXR];
  out->min_p = h[ST_MINP];
  out->max_p = h[ST_MAXP];
  return MLBM_OK;
}

static_assert(ST_COUNT + 1 == MLBM_STATS_RAW_LEN, "raw statistics length");

}  // namespace

extern "C" {

mlbm_status mlbm_phase_stats(mlbm_lattice* lat, mlbm_stats* out) {
  if (!out) return fail(MLBM_ERR_ARG, "null output");
  double h[ST_COUNT + 1];
  if (mlbm_status st = stats_enqueue(lat, h, true)) return st;
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "stats");
  return stats_convert(lat, h, out);
}

mlbm_status mlbm_phase_stats_async(mlbm_lattice* lat, double* raw) {
  return stats_enqueue(lat, raw, true);
}

mlbm_status mlbm_bulk_stats_async(mlbm_lattice* lat, double* raw) {
  return stats_enqueue(lat, raw, false);
}

mlbm_status mlbm_stats_from_raw(mlbm_lattice* lat, const double* raw,
                                mlbm_stats* out) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!raw || !out) return fail(MLBM_ERR_ARG, "null argument");
  return stats_convert(lat, raw, out);
}

mlbm_status mlbm_plane_profile(mlbm_lattice* lat, int64_t* n_fluid_x,
                               int64_t* n_liquid_x) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!n_fluid_x || !n_liquid_x) return fail(MLBM_ERR_ARG, "null output");
  if (!lat->initialized) return fail(MLBM_ERR_STATE, "profile before initialize");
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  const int lx = lat->g.lx;
  const size_t bytes = 2 * (size_t)lx * sizeof(unsigned long long);
  if (mlbm_status st = ensure_staging(lat, bytes)) return st;
  auto* nf = static_cast<unsigned long long*>(lat->staging);
  auto* nl = nf + lx;
  CUDA_TRY(cudaMemsetAsync(nf, 0, bytes, lat->stream), "profile clear");
  if (lat->storage == MLBM_STORE_F64)
    k_plane_profile<double><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        static_cast<const double*>(lat->rho), lat->mask, lat->g, lat->phys, nf, nl);
  else
    k_plane_profile<float><<<node_grid(lat->g), node_block(), 0, lat->stream>>>(
        static_cast<const float*>(lat->rho), lat->mask, lat->g, lat->phys, nf, nl);
  CUDA_TRY(cudaGetLastError(), "profile launch");
  CUDA_TRY(cudaMemcpyAsync(n_fluid_x, nf, lx * 8, cudaMemcpyDeviceToHost,
                           lat->stream), "profile copy");
  CUDA_TRY(cudaMemcpyAsync(n_liquid_x, nl, lx * 8, cudaMemcpyDeviceToHost,
                           lat->stream), "profile copy");
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "profile");
  return MLBM_OK;
}

mlbm_status mlbm_set_step_kernel(mlbm_lattice* lat, int32_t kind) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (kind != MLBM_KERNEL_AUTO && kind != MLBM_KERNEL_TWO_PASS &&
      kind != MLBM_KERNEL_COMPACT && kind != MLBM_KERNEL_BAND)
    return fail(MLBM_ERR_ARG, "invalid step kernel %d", kind);
  if (kind == MLBM_KERNEL_BAND && !compact_band_supported(lat))
    return fail(MLBM_ERR_ARG,
                "one-pass step needs FP32 or FP16 storage, at most 2048 x 2048 "
                "x 1024 nodes and a whole lattice (not a slab)");
  if (kind == MLBM_KERNEL_COMPACT && !lat->compact.two_pass_ok)
    return fail(MLBM_ERR_ARG,
                "compact kernels need FP32 or FP16 storage and at most "
                "2048 x 2048 x 1024 nodes");
  lat->step_kernel = kind;
  return MLBM_OK;
}

mlbm_status mlbm_set_update_shape(mlbm_lattice* lat, int32_t rows,
                                  int32_t planes) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (rows < 1 || rows > 8 || planes < 1 || planes > 1024)
    return fail(MLBM_ERR_ARG, "invalid update shape %d x %d", rows, planes);
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "update shape");
  return setup_update(lat, rows, planes);
}

int32_t mlbm_get_step_kernel(const mlbm_lattice* lat) {
  return lat ? effective_kernel(lat) : -1;
}

mlbm_status mlbm_set_wait_limit(mlbm_lattice* lat, uint64_t ns) {
  if (mlbm_status st = check_lat(lat)) return st;
  lat->wait_ns = ns ? ns : kDefaultWaitNs;
  return MLBM_OK;
}

mlbm_status mlbm_test_stall_wait(mlbm_lattice* lat) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (effective_kernel(lat) != MLBM_KERNEL_BAND)
    return fail(MLBM_ERR_STATE,
                "test_stall_wait: the lattice's step kernel has no such wait "
                "(select MLBM_KERNEL_BAND)");
  lat->stall_test = true;
  return MLBM_OK;
}

mlbm_status mlbm_set_band_shape(mlbm_lattice* lat, int32_t rows,
                                int32_t planes) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (rows < 1 || rows > 64 || planes < 1 || planes > 1024)
    return fail(MLBM_ERR_ARG, "invalid one-pass shape %d rows x %d planes",
                rows, planes);
  return compact_set_band_shape(lat, rows, planes);
}

mlbm_status mlbm_autotune(mlbm_lattice* lat, int64_t step0,
                          int32_t trial_steps, int32_t* out,
                          int32_t* steps_done) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (!lat->initialized) return fail(MLBM_ERR_STATE, "autotune before initialize");
  if (trial_steps < 1) trial_steps = 2;
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  if (effective_kernel(lat) == MLBM_KERNEL_COMPACT) {
    // one thread per fluid node: nothing to tune
    if (out) out[0] = out[1] = 0;
    if (steps_done) *steps_done = 0;
    return MLBM_OK;
  }
  const bool band = effective_kernel(lat) == MLBM_KERNEL_BAND;
  const int rows_u[] = {1, 2, 4, 8};
  const int planes_u[] = {2, 4, 8, 16, 32};
  // one-pass step: rows per band x planes per chunk
  const int rows_b[] = {2, 4, 6, 8};
  const int planes_b[] = {8, 16, 24, 32, 48};
  const int* rows_c = band ? rows_b : rows_u;
  const int* planes_c = band ? planes_b : planes_u;
  const int nr = 4, np = 5;
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0), "autotune");
  CUDA_TRY(cudaEventCreate(&e1), "autotune");
  float best = 1e30f;
  int br = band ? lat->compact.band_rows : lat->zm.By;
  int bp = band ? lat->compact.band_planes : lat->zm.Dz;
  auto apply = [&](int r, int pl) -> mlbm_status {
    if (band) return compact_set_band_shape(lat, r, pl);
    return setup_update(lat, r, pl);
  };
  int64_t step = step0;
  for (int ri = 0; ri < nr; ++ri)
    for (int pi = 0; pi < np; ++pi) {
      const int r = rows_c[ri], pl = planes_c[pi];
      if (apply(r, pl) != MLBM_OK) continue;
      if (mlbm_status st = mlbm_iterate(lat, step, 1, 1, 0, 0)) return st;
      step += 1;
      cudaEventRecord(e0, lat->stream);
      if (mlbm_status st = mlbm_iterate(lat, step, trial_steps, 1, 0, 0)) return st;
      step += trial_steps;
      cudaEventRecord(e1, lat->stream);
      CUDA_TRY(cudaEventSynchronize(e1), "autotune");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        br = r;
        bp = pl;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (mlbm_status st = apply(br, bp)) return st;
  if (out) {
    out[0] = br;
    out[1] = bp;
  }
  if (steps_done) *steps_done = (int32_t)(step - step0);
  return MLBM_OK;
}

mlbm_status mlbm_synchronize(mlbm_lattice* lat) {
  if (mlbm_status st = check_lat(lat)) return st;
  DeviceGuard restore_device;
  if (mlbm_status st = activate(lat)) return st;
  CUDA_TRY(cudaStreamSynchronize(lat->stream), "synchronize");
  return check_device_error(lat);
}

mlbm_status mlbm_lattice_info(const mlbm_lattice* lat, int32_t* dims,
                              int32_t* storage, int32_t* phase,
                              int32_t* initialized) {
  if (mlbm_status st = check_lat(lat)) return st;
  if (dims) {
    dims[0] = lat->g.lx;
    dims[1] = lat->g.ly;
    dims[2] = lat->g.lz;
  }
  if (storage) *storage = lat->storage;
  if (phase) *phase = lat->phase;
  if (initialized) *initialized = lat->initialized ? 1 : 0;
  return MLBM_OK;
}

}  // extern "C"
