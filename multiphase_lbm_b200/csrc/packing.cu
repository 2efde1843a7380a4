// packing.cu -- the seeded sphere packing of mlbm_generate_packing, with the
// voxelisation on the GPU (include/mlbm_host.h, mlbm_generate_packing_gpu).
//
// The host generator places spheres one after the other until the porosity
// reaches the target, counting the nodes each sphere turns solid.  The same
// result without the sequence: voxelise a chunk of candidate spheres (drawn
// from the same SplitMix64 stream) at once, keeping for every node the index
// of the FIRST sphere that covers it (atomicMin); the nodes sphere j turns
// solid are exactly the nodes whose first sphere is j.  A prefix sum over j
// then finds the first sphere after which the porosity is at or below the
// target, and the mask is "first sphere index <= that sphere".  Candidates
// come in chunks until the target is reached or max_spheres is spent.
//
// Every sphere is voxelised as the reference's place_sphere does
// (src/multiphase_lbm.cu:893-927): coordinates advanced from x - R by
// repeated float additions of 1.0, the float distance test
// (dx*dx + dy*dy) + dz*dz < R*R with every operation rounded on its own,
// nearest() = floor(v + 0.5) in double, one periodic wrap (repeated for
// spheres larger than the box).  The mask is bit-identical to the host's.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mlbm_host.h"
#include "errors.h"
#include "host/splitmix.h"

namespace mlbm {
namespace {

__device__ __forceinline__ int pk_nearest(float v) {
  return (int)floor((double)v + 0.5);
}
__device__ __forceinline__ int pk_wrap(int v, int n) {
  while (v < 0) v += n;
  while (v >= n) v -= n;
  return v;
}

// One block per candidate sphere: thread (i, j) walks the pz line of the i-th
// px and j-th py position of the footprint (32 x 32 threads, strided for
// larger spheres).
__global__ void k_first_cover(const float4* __restrict__ spheres, int base,
                              int n, int lx, int ly, int lz,
                              unsigned* __restrict__ first) {
  const int s = blockIdx.x;
  if (s >= n) return;
  const float4 c = spheres[s];
  const float x = c.x, y = c.y, z = c.z, R = c.w;
  const float xmin = __fsub_rn(x, R), ymin = __fsub_rn(y, R), zmin = __fsub_rn(z, R);
  const float xmax = __fadd_rn(x, R), ymax = __fadd_rn(y, R), zmax = __fadd_rn(z, R);
  const float R2 = __fmul_rn(R, R);
  const unsigned id = (unsigned)(base + s);
  for (int i = threadIdx.x;; i += blockDim.x) {
    float px = xmin;
    for (int t = 0; t < i; ++t) px = __fadd_rn(px, 1.0f);
    if (!(px <= xmax)) break;
    const float dx = __fsub_rn(px, x);
    const float dxx = __fmul_rn(dx, dx);
    const int nx = pk_wrap(pk_nearest(px), lx);
    for (int j = threadIdx.y;; j += blockDim.y) {
      float py = ymin;
      for (int t = 0; t < j; ++t) py = __fadd_rn(py, 1.0f);
      if (!(py <= ymax)) break;
      const float dy = __fsub_rn(py, y);
      const float dxy = __fadd_rn(dxx, __fmul_rn(dy, dy));
      const int ny = pk_wrap(pk_nearest(py), ly);
      const long long row = ((long long)nx * ly + ny) * lz;
      for (float pz = zmin; pz <= zmax; pz = __fadd_rn(pz, 1.0f)) {
        const float dz = __fsub_rn(pz, z);
        if (__fadd_rn(dxy, __fmul_rn(dz, dz)) < R2)
          atomicMin(first + row + pk_wrap(pk_nearest(pz), lz), id);
      }
    }
  }
}

// Nodes each sphere of [base, base + n) covers first (integer atomics).
__global__ void k_count_first(const unsigned* __restrict__ first, long long total,
                              int base, int n,
                              unsigned long long* __restrict__ flips) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  const unsigned f = first[k];
  if (f != UINT_MAX && (int)f >= base && (int)f < base + n)
    atomicAdd(flips + ((int)f - base), 1ull);
}

// Solid where the first covering sphere is one of the `placed` placed ones.
__global__ void k_mask_from_first(const unsigned* __restrict__ first,
                                  long long total, long long placed,
                                  uint8_t* __restrict__ is_fluid) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  is_fluid[k] = (long long)first[k] < placed ? 0 : 1;
}

mlbm_status cuda_fail(cudaError_t e, const char* where) {
  cudaGetLastError();
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
  return set_error(MLBM_ERR_CUDA, msg);
}

struct Buffers {
  unsigned* first = nullptr;
  float4* spheres = nullptr;
  unsigned long long* flips = nullptr;
  uint8_t* mask = nullptr;
  ~Buffers() {
    cudaFree(first);
    cudaFree(spheres);
    cudaFree(flips);
    cudaFree(mask);
  }
};

}  // namespace
}  // namespace mlbm

using namespace mlbm;

extern "C" mlbm_status mlbm_generate_packing_gpu(
    int32_t lx, int32_t ly, int32_t lz, float rmin, float rmax,
    double porosity_target, uint64_t seed, int64_t max_spheres,
    int32_t device, uint8_t* is_fluid, float* xyzr, int64_t* count,
    double* porosity) {
  if (!is_fluid || lx < 1 || ly < 1 || lz < 1 || !(rmin > 0.f) ||
      !(rmax >= rmin) || max_spheres < 0)
    return set_error(MLBM_ERR_ARG, "generate_packing_gpu: bad arguments");
  const long long n = (long long)lx * ly * lz;
  if (max_spheres >= (int64_t)UINT_MAX)
    return set_error(MLBM_ERR_ARG, "generate_packing_gpu: too many spheres");
  mlbm::DeviceGuard restore_device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu");
  Buffers b;
  // candidates per chunk: about what the target takes, from the mean
  // sphere volume (overlap makes it more; later chunks double)
  const double rm = 0.5 * (rmin + rmax);
  const double vol = 4.18879 * rm * rm * rm;
  long long chunk = std::max<long long>(
      64, (long long)(1.2 * (1.0 - porosity_target) * n / std::max(vol, 1.0)));
  const long long cap = std::max<long long>(chunk, 1 << 16);
  e = cudaMalloc((void**)&b.first, n * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(b.first, 0xff, n * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b.spheres, cap * sizeof(float4));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&b.flips, cap * sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu buffers");
  SplitMix64 rng{seed};
  std::vector<float4> cand;
  std::vector<unsigned long long> flips;
  long long fluid = n, placed = 0;
  bool done = (double)fluid / (double)n <= porosity_target || max_spheres == 0;
  while (!done) {
    const long long m = std::min<long long>({chunk, cap, max_spheres - placed});
    cand.resize(m);
    for (long long j = 0; j < m; ++j) {
      const float cx = rng.uniform() * (float)lx;
      const float cy = rng.uniform() * (float)ly;
      const float cz = rng.uniform() * (float)lz;
      const float r = rmin + rng.uniform() * (rmax - rmin);
      cand[j] = make_float4(cx, cy, cz, r);
    }
    e = cudaMemcpy(b.spheres, cand.data(), m * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemset(b.flips, 0, m * sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu");
    k_first_cover<<<(unsigned)m, dim3(32, 32)>>>(b.spheres, (int)placed, (int)m,
                                                 lx, ly, lz, b.first);
    k_count_first<<<(unsigned)((n + 255) / 256), 256>>>(b.first, n, (int)placed,
                                                         (int)m, b.flips);
    flips.resize(m);
    e = cudaMemcpy(flips.data(), b.flips, m * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu");
    for (long long j = 0; j < m && !done; ++j) {
      fluid -= (long long)flips[j];
      if (xyzr) {
        xyzr[4 * (placed + j)] = cand[j].x;
        xyzr[4 * (placed + j) + 1] = cand[j].y;
        xyzr[4 * (placed + j) + 2] = cand[j].z;
        xyzr[4 * (placed + j) + 3] = cand[j].w;
      }
      if ((double)fluid / (double)n <= porosity_target ||
          placed + j + 1 >= max_spheres) {
        placed += j + 1;
        done = true;
      }
    }
    if (!done) {
      placed += m;
      chunk = std::min<long long>(2 * chunk, cap);
    }
  }
  // the spheres after the last placed one of the final chunk covered nodes
  // too: the mask keeps only first covers by spheres 0 .. placed - 1
  e = cudaMalloc((void**)&b.mask, n);
  if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu mask");
  k_mask_from_first<<<(unsigned)((n + 255) / 256), 256>>>(b.first, n, placed,
                                                           b.mask);
  e = cudaMemcpy(is_fluid, b.mask, n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "generate_packing_gpu");
  if (count) *count = placed;
  if (porosity) *porosity = (double)fluid / (double)n;
  return MLBM_OK;
}
