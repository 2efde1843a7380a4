// persistent.cu -- host side of the fused z-marching time step
// (persistent.cuh): tile-shape choice, occupancy-checked cooperative launch,
// progress counters.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

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

size_t window_bytes(int Tx, int Ty, int storage) {
  return (size_t)3 * (Tx + 2) * (Ty + 2) * real_bytes(storage);
}

// Blocks of `fn` that fit one SM at this block size and shared memory.
int blocks_per_sm(const void* fn, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace

int max_tiles(const Geom& g) { return (g.px / 32) * g.ly; }

FusedShape fused_shape(const Geom& g, int storage, int ty_hint, int lag) {
  FusedShape f{};
  f.Tx = 32;
  f.Ty = std::max(1, std::min(ty_hint > 0 ? ty_hint : 0, 16));
  f.L = std::max(2, lag > 0 ? lag : 4);
  f.ok = true;
  f.chosen = ty_hint > 0;  // otherwise chosen at the first launch
  if (f.chosen) {
    f.Ty = std::min(f.Ty, g.ly);
    f.ntx = g.px / f.Tx;
    f.nty = (g.ly + f.Ty - 1) / f.Ty;
    f.ntiles = f.ntx * f.nty;
    f.threads = f.Tx * f.Ty;
    f.smem = window_bytes(f.Tx, f.Ty, storage);
  }
  return f;
}

// Pick the tile (Tx = 32 x Ty) for this lattice: every tile's block must be
// co-resident (the grid is one block per tile); among those, prefer an even
// number of blocks per SM, then the smaller psi halo.
template <typename T>
mlbm_status choose_tiles(mlbm_lattice* lat) {
  FusedShape& f = lat->fused;
  const Geom& g = lat->g;
  int nsm = 0;
  cudaError_t e =
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, lat->device);
  if (e != cudaSuccess) return cuda_fail(e, "SM count");
  // the heaviest variant bounds the occupancy of all of them
  const void* fn = pick_fn<T>(0, OUT_RHO | OUT_VEL);
  double best = -1.0;
  int best_ty = 0;
  const int tys[] = {1, 2, 4, 8, 16};
  for (int ty : tys) {
    if (f.chosen && ty != f.Ty) continue;
    if (ty > g.ly && ty != 1) continue;
    const int threads = 32 * ty;
    const int ntiles = (g.px / 32) * ((g.ly + ty - 1) / ty);
    const int per_sm = blocks_per_sm(fn, threads, window_bytes(32, ty, lat->storage));
    if (per_sm < 1 || ntiles > per_sm * nsm) continue;
    const int rounds = (ntiles + nsm - 1) / nsm;
    const double balance = (double)ntiles / ((double)nsm * rounds);
    const double halo = (34.0 * (ty + 2)) / (32.0 * ty);
    const double score = std::floor(balance * 50.0) - 0.5 * halo;
    if (score > best) {
      best = score;
      best_ty = ty;
    }
  }
  if (best_ty == 0) {
    f.ok = false;
    return set_error(MLBM_ERR_ARG,
                     "fused kernel: the lattice has more tiles than the GPU "
                     "holds blocks at once");
  }
  f.Ty = best_ty;
  f.ntx = g.px / 32;
  f.nty = (g.ly + f.Ty - 1) / f.Ty;
  f.ntiles = f.ntx * f.nty;
  f.threads = 32 * f.Ty;
  f.smem = window_bytes(32, f.Ty, lat->storage);
  f.chosen = true;
  return MLBM_OK;
}

template <typename T>
mlbm_status launch_fused(mlbm_lattice* lat, const StepArgs& a, int out) {
  using R = typename Pop<T>::Real;
  if (!lat->fused.chosen || lat->fused.ntiles == 0)
    if (mlbm_status st = choose_tiles<T>(lat)) return st;
  const FusedShape& fs = lat->fused;
  const void* fn = pick_fn<T>(lat->phase, out);
  // Counters are cumulative over launches (each launch adds lz); restart
  // them before they could wrap.
  if (lat->fused_epoch + 2ull * (unsigned)lat->g.lz >= (1ull << 31)) {
    cudaError_t e = cudaMemsetAsync(lat->pdone, 0,
                                    sizeof(unsigned) * max_tiles(lat->g),
                                    lat->stream);
    if (e != cudaSuccess) return cuda_fail(e, "counter reset");
    lat->fused_epoch = 0;
  }
  March s;
  s.Tx = fs.Tx;
  s.Ty = fs.Ty;
  s.ntx = fs.ntx;
  s.nty = fs.nty;
  s.L = fs.L;
  s.base = (unsigned)lat->fused_epoch;
  s.budget_cycles = 1LL << 32;  // about 2 s at B200 clocks

  T* pop = static_cast<T*>(lat->pop);
  R* psi = static_cast<R*>(lat->psi);
  R* rho = static_cast<R*>(lat->rho);
  float* vel = lat->vel;
  const uint32_t* nbw = lat->nbw;
  unsigned* prog = lat->pdone;
  int* err = lat->err;
  Geom g = lat->g;
  Phys p = lat->phys;
  StepArgs aa = a;
  void* args[] = {&pop, &nbw, &psi, &rho, &vel, &prog, &err, &g, &p, &aa, &s};
  cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(fs.ntiles),
                                              dim3(fs.threads), args, fs.smem,
                                              lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "fused time-step launch");
  lat->fused_epoch += (unsigned)lat->g.lz;
  return MLBM_OK;
}

template mlbm_status launch_fused<float>(mlbm_lattice*, const StepArgs&, int);
template mlbm_status launch_fused<__half>(mlbm_lattice*, const StepArgs&, int);
template mlbm_status launch_fused<double>(mlbm_lattice*, const StepArgs&, int);

}  // namespace mlbm
