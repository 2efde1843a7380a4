// noalloc.cu -- mlbm_phase_stats_noalloc: the phase statistics of
// mlbm_phase_stats computed without allocating any memory.
//
// Who needs it: callers that cannot call cudaMalloc when they want
// statistics -- an application that reserves the GPU's memory up front for
// its own pool (a library's cudaMalloc would then fail, or take memory the
// pool has promised elsewhere), and solver loops embedded in a host that
// forbids libraries to allocate because cudaMalloc and cudaFree may
// synchronise the device and take unbounded time.  They pass device pointers
// to fields they already own; this entry point adds no allocation of its own
// (no cudaMalloc, cudaFree or allocating library routine).  It does copy the
// result row to a host array and waits for the caller's stream before it
// returns.
//
// Its scratch -- one row of partial sums per x-plane plus one result row --
// lives in a file-scope __device__ array of fixed size.  Every GPU that loads
// libmlbm holds it (about 459 KB) until the process exits.  Its size caps the
// lattice at MLBM_NOALLOC_MAX_LX planes in x; larger lattices are rejected
// with MLBM_ERR_ARG.  All calls share the array: two calls that overlap on
// the GPU (different streams, or different host threads) race on it and
// corrupt each other's results, so serialise them.  Each call writes every
// row it later reads, so nothing left by a previous call is ever used and
// nothing needs clearing.
//
// In host code the array's name is only a host-side stand-in, not a device
// address.  The first call on each device therefore looks the real address
// up with cudaGetSymbolAddress (with that device current) and keeps it; that
// lookup may load the library's device code, so a caller that restricts
// which CUDA calls may run at a given point makes the first call during its
// setup.  The kept
// address belongs to the device's primary context: a process that resets
// the device (cudaDeviceReset) must not call this entry point afterwards.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/mlbm.h"
#include "errors.h"
#include "lattice.cuh"

namespace {

// Slots of one row of partial results.
enum { ST_NF, ST_NL, ST_NV, ST_NLS, ST_NLV, ST_MASS, ST_PL, ST_PV, ST_RL,
       ST_RV, ST_MINR, ST_MAXR, ST_MINP, ST_MAXP, ST_COUNT };

constexpr int kMaxLx = MLBM_NOALLOC_MAX_LX;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

// Rows 0 .. lx-1: partial results of x-plane x; row kMaxLx: the final row.
static __device__ __align__(256) double
    g_noalloc_scratch[(kMaxLx + 1) * ST_COUNT];

std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {nullptr};

__device__ __forceinline__ double combine(int k, double a, double b) {
  return (k == ST_MINR || k == ST_MINP) ? fmin(a, b)
         : (k == ST_MAXR || k == ST_MAXP) ? fmax(a, b)
                                           : a + b;
}

// One block per x-plane of the reference layout [x][y][z]: the plane is the
// contiguous run of ly*lz values starting at x*ly*lz.  Same statistics as
// k_stats_partial (src/multiphase_lbm.cu:240-316, 1061-1072).
__global__ void __launch_bounds__(kThreads)
    k_stats_plane_ref(const float* __restrict__ rho,
                      const uint8_t* __restrict__ fluid, int lx, int ly,
                      int lz, mlbm::Phys p, double* __restrict__ scratch) {
  using namespace mlbm;
  const int x = blockIdx.x;
  const long long plane = (long long)ly * lz;
  double acc[ST_COUNT];
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) acc[k] = 0.0;
  acc[ST_MINR] = 1e9;
  acc[ST_MAXR] = -1e-9;
  acc[ST_MINP] = 1e9;
  acc[ST_MAXP] = -1e-9;
  const float rhol = p.rhol_spinodal, rhog = p.rhog_spinodal;
  for (long long j = threadIdx.x; j < plane; j += blockDim.x) {
    const long long k = x * plane + j;
    if (!fluid[k]) continue;
    const int y = (int)(j / lz), z = (int)(j % lz);
    const float r = rho[k];
    const float pr = pressure_of<float>(p, r);
    acc[ST_NF] += 1.0;
    acc[ST_MASS] += (double)r;
    if (r > rhol) {
      acc[ST_NL] += 1.0;
      acc[ST_PL] += (double)pr;
      acc[ST_RL] += (double)r;
      for (int i = 1; i < Q; ++i) {
        const int xn = wrapc(x - ex(i), lx), yn = wrapc(y - ey(i), ly),
                  zn = wrapc(z - ez(i), lz);
        const long long kn = ((long long)xn * ly + yn) * lz + zn;
        if (!fluid[kn]) { acc[ST_NLS] += 1.0; break; }
        if (rho[kn] < rhol) { acc[ST_NLV] += 1.0; break; }
      }
    } else if (r < rhog) {
      acc[ST_NV] += 1.0;
      acc[ST_PV] += (double)pr;
      acc[ST_RV] += (double)r;
    }
    acc[ST_MINR] = fmin(acc[ST_MINR], (double)r);
    acc[ST_MAXR] = fmax(acc[ST_MAXR], (double)r);
    acc[ST_MINP] = fmin(acc[ST_MINP], (double)pr);
    acc[ST_MAXP] = fmax(acc[ST_MAXP], (double)pr);
  }
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) {
    double v = acc[k];
    for (int off = 16; off > 0; off >>= 1)
      v = combine(k, v, __shfl_down_sync(0xffffffffu, v, off));
    acc[k] = v;
  }
  __shared__ double sh[kThreads / 32][ST_COUNT];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < ST_COUNT; ++k) sh[warp][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < ST_COUNT) {
    const int k = threadIdx.x;
    double v = sh[0][k];
    for (int w = 1; w < kThreads / 32; ++w) v = combine(k, v, sh[w][k]);
    scratch[(long long)x * ST_COUNT + k] = v;
  }
}

// Fold the lx plane rows in plane order into the final row (deterministic).
__global__ void k_stats_plane_final(int lx, double* __restrict__ scratch) {
  const int k = threadIdx.x;
  if (k >= ST_COUNT) return;
  double v = scratch[k];
  for (int x = 1; x < lx; ++x) v = combine(k, v, scratch[(long long)x * ST_COUNT + k]);
  scratch[(long long)kMaxLx * ST_COUNT + k] = v;
}

mlbm_status scratch_for_device(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices)
    return mlbm::set_error(MLBM_ERR_CUDA, "phase_stats_noalloc: device id out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return mlbm::set_error(MLBM_ERR_CUDA,
                             "phase_stats_noalloc: cudaGetSymbolAddress failed");
    }
    g_scratch_addr[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_addr[dev];
  return MLBM_OK;
}

}  // namespace

extern "C" mlbm_status mlbm_phase_stats_noalloc(
    const float* rho_dev, const uint8_t* is_fluid_dev, int32_t lx, int32_t ly,
    int32_t lz, const mlbm_params* params, void* stream, mlbm_stats* out) {
  using namespace mlbm;
  if (!rho_dev || !is_fluid_dev || !params || !out)
    return set_error(MLBM_ERR_ARG, "phase_stats_noalloc: null argument");
  if (lx < 1 || ly < 1 || lz < 1)
    return set_error(MLBM_ERR_ARG, "phase_stats_noalloc: invalid lattice size");
  if (lx > kMaxLx)
    return set_error(MLBM_ERR_ARG,
                     "phase_stats_noalloc: lx exceeds MLBM_NOALLOC_MAX_LX "
                     "(the size of the static scratch array)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_error(MLBM_ERR_CUDA, "phase_stats_noalloc: no current device");
  }
  double* scratch = nullptr;
  if (mlbm_status st = scratch_for_device(dev, &scratch)) return st;

  Phys p;
  std::memset(&p, 0, sizeof p);
  p.G = params->G;
  p.T_Tc = params->T_Tc;
  p.carn_star = params->carn_star;
  p.rhol_spinodal = params->rhol_spinodal;
  p.rhog_spinodal = params->rhog_spinodal;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_stats_plane_ref<<<lx, kThreads, 0, s>>>(rho_dev, is_fluid_dev, lx, ly, lz,
                                            p, scratch);
  k_stats_plane_final<<<1, 32, 0, s>>>(lx, scratch);
  cudaError_t e = cudaGetLastError();
  double h[ST_COUNT];
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, scratch + (size_t)kMaxLx * ST_COUNT, sizeof h,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return set_error(MLBM_ERR_CUDA, cudaGetErrorString(e));

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
