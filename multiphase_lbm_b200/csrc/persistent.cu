// persistent.cu -- host side of the fused persistent time step
// (persistent.cuh): schedule geometry, occupancy-sized cooperative launch,
// error-flag handling.
#include <cuda_runtime.h>

#include <algorithm>

#include "capi_internal.h"
#include "persistent.cuh"

namespace mlbm {

namespace {

template <typename T, int PHASE, int OUT>
const void* fused_fn() {
  return reinterpret_cast<const void*>(&k_step_fused<T, PHASE, OUT>);
}

template <typename T>
const void* pick_fn(int phase, int out) {
  if (phase == 0) {
    switch (out) {
      case OUT_NONE: return fused_fn<T, 0, OUT_NONE>();
      case OUT_RHO: return fused_fn<T, 0, OUT_RHO>();
      default: return fused_fn<T, 0, OUT_RHO | OUT_VEL>();
    }
  }
  switch (out) {
    case OUT_NONE: return fused_fn<T, 1, OUT_NONE>();
    case OUT_RHO: return fused_fn<T, 1, OUT_RHO>();
    default: return fused_fn<T, 1, OUT_RHO | OUT_VEL>();
  }
}

}  // namespace

FusedShape fused_shape(const Geom& g, int storage, int by_hint, int lag) {
  FusedShape f{};
  f.nseg = (g.px + 511) / 512;
  f.W = ((g.px / 32 + f.nseg - 1) / f.nseg) * 32;
  int by = by_hint > 0 ? by_hint : std::max(1, 256 / f.W);
  by = std::min(by, std::max(1, 512 / f.W));
  by = std::min(by, g.ly);
  f.By = by;
  f.threads = f.By * f.W;
  f.rb_y = (g.ly + f.By - 1) / f.By;
  f.R = f.rb_y * f.nseg;
  f.L = std::max(2, std::min(lag > 0 ? lag : 4, g.lz));
  if (f.L > g.lz) f.L = g.lz;
  f.smem = (size_t)3 * (f.By + 2) * g.lx * real_bytes(storage);
  f.ok = f.smem <= 160 * 1024 && f.threads <= 512;
  return f;
}

template <typename T>
mlbm_status launch_fused(mlbm_lattice* lat, const StepArgs& a, int out) {
  using R = typename Pop<T>::Real;
  const FusedShape& fs = lat->fused;
  const void* fn = pick_fn<T>(lat->phase, out);
  const int key = lat->phase * 3 + (out == OUT_NONE ? 0 : (out == OUT_RHO ? 1 : 2));
  if (lat->fused_grid[key] == 0) {
    if (fs.smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(
          fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fs.smem);
      if (e != cudaSuccess) return cuda_fail(e, "fused kernel smem attribute");
    }
    int per_sm = 0, nsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, fn, fs.threads, fs.smem);
    if (e != cudaSuccess) return cuda_fail(e, "fused kernel occupancy");
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, lat->device);
    if (e != cudaSuccess) return cuda_fail(e, "SM count");
    if (per_sm < 1) return set_error(MLBM_ERR_CUDA, "fused kernel does not fit an SM");
    lat->fused_grid[key] = per_sm * nsm;
  }
  // Counters are cumulative; reset them before the target would overflow.
  if ((unsigned long long)(lat->fused_epoch + 2) * (unsigned)fs.R >= (1ull << 31)) {
    cudaError_t e = cudaMemsetAsync(lat->pdone, 0, sizeof(unsigned) * lat->g.lz,
                                    lat->stream);
    if (e != cudaSuccess) return cuda_fail(e, "counter reset");
    lat->fused_epoch = 0;
  }
  Sched s;
  s.By = fs.By;
  s.W = fs.W;
  s.nseg = fs.nseg;
  s.rb_y = fs.rb_y;
  s.R = fs.R;
  s.L = fs.L;
  s.total = 2LL * lat->g.lz * fs.R;
  s.target = (unsigned)((lat->fused_epoch + 1) * (unsigned long long)fs.R);
  s.budget_cycles = 1LL << 32;  // about 2 s at B200 clocks
  const long long want = s.total;
  const int grid = (int)std::min<long long>(lat->fused_grid[key], want);

  T* pop = static_cast<T*>(lat->pop);
  R* psi = static_cast<R*>(lat->psi);
  R* rho = static_cast<R*>(lat->rho);
  float* vel = lat->vel;
  const uint32_t* nbw = lat->nbw;
  unsigned* pdone = lat->pdone;
  int* err = lat->err;
  Geom g = lat->g;
  Phys p = lat->phys;
  StepArgs aa = a;
  void* args[] = {&pop, &nbw, &psi, &rho, &vel, &pdone, &err, &g, &p, &aa, &s};
  cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(fs.threads),
                                              args, fs.smem, lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "fused time-step launch");
  lat->fused_epoch += 1;
  return MLBM_OK;
}

template mlbm_status launch_fused<float>(mlbm_lattice*, const StepArgs&, int);
template mlbm_status launch_fused<__half>(mlbm_lattice*, const StepArgs&, int);
template mlbm_status launch_fused<double>(mlbm_lattice*, const StepArgs&, int);

}  // namespace mlbm
