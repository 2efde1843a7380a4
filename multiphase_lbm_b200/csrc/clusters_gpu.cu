// clusters_gpu.cu -- the cluster statistics of calc_cluster
// (src/multiphase_lbm.cu:225-562) on the GPU (mlbm_cluster_stats_gpu,
// include/mlbm_driver.h); the same results as the host mlbm_cluster_stats.
//
// Clusters are the 6-connected (periodic) components of the liquid nodes
// (rho > rhol_spinodal) and of the gas nodes (rho < rhog_spinodal) among the
// fluid nodes.  The reference floods them with a recursive depth-first
// search in its x-major scan order and numbers them by their first node in
// that order, dropping clusters of fewer than 7 nodes.  Here a lock-free
// union-find links every node to the smallest reference index of its
// component (atomicMin linking, then path flattening), so the root of a
// cluster IS its first node in the scan; a prefix count of the kept roots
// (size >= 7) in index order gives the reference's cluster numbers.
//
// The other columns:
//   liquid-solid / liquid-vapour boundary counts -- the first of the 18
//     neighbours x - e_i that is solid or not liquid decides (:278-316);
//   cluster order and wet coordination number (:535-561) -- both depend only
//     on the distinct (liquid cluster, solid number) pairs of 6-neighbours:
//     order = pairs / clusters touching a solid (0/0 = NaN when none does,
//     as in the reference), wet = pairs / solid_count; the pairs are sorted
//     on the device and counted;
//   single-cluster radius (:362-533) -- periodic unwrapping tests, the first
//     free planes, integer-divided centre and the largest distance, with the
//     host code's float arithmetic (each operation rounded on its own).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mlbm_driver.h"
#include "errors.h"

namespace mlbm {
namespace {

constexpr int kMinCluster = 7;  // src/multiphase_lbm.cu:321

// D3Q19 velocities, include/lbm_model.cuh:49-54
__constant__ int c_ex[19] = {0, -1, 0, 0, -1, -1, -1, -1, 0, 0, 1, 0, 0, 1, 1, 1, 1, 0, 0};
__constant__ int c_ey[19] = {0, 0, -1, 0, -1, 1, 0, 0, -1, -1, 0, 1, 0, 1, -1, 0, 0, 1, 1};
__constant__ int c_ez[19] = {0, 0, 0, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, 0, 0, 1, -1, 1, -1};

struct Dims {
  int lx, ly, lz;
  long long n;
  __device__ __forceinline__ long long idx(int x, int y, int z) const {
    return ((long long)x * ly + y) * lz + z;
  }
  __device__ __forceinline__ void xyz(long long k, int& x, int& y, int& z) const {
    z = (int)(k % lz);
    const long long r = k / lz;
    y = (int)(r % ly);
    x = (int)(r / ly);
  }
};

// class: 1 liquid, 2 gas, 0 neither (solid or in between)
__global__ void k_classify(const float* __restrict__ rho,
                           const uint8_t* __restrict__ fluid, Dims d,
                           float rhol, float rhog, uint8_t* __restrict__ cls,
                           int* __restrict__ parent) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  uint8_t c = 0;
  if (fluid[k]) {
    const float r = rho[k];
    c = r > rhol ? 1 : (r < rhog ? 2 : 0);
  }
  cls[k] = c;
  parent[k] = (int)k;
}

__device__ __forceinline__ int uf_find(const int* parent, int a) {
  int p = parent[a];
  while (p != a) {
    a = p;
    p = parent[a];
  }
  return a;
}

// Link the roots of a and b, the larger under the smaller, until they agree.
__device__ __forceinline__ void uf_unite(int* parent, int a, int b) {
  for (;;) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(parent + b, a);
    if (old == b) return;  // b was a root and now hangs under a
    b = old;               // b gained a smaller parent meanwhile: retry
  }
}

// Each node unites with its +x, +y, +z neighbours (periodic) of its class.
__global__ void k_unite(const uint8_t* __restrict__ cls, Dims d,
                        int* __restrict__ parent) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  const uint8_t c = cls[k];
  if (!c) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  const long long q[3] = {d.idx(x + 1 < d.lx ? x + 1 : 0, y, z),
                          d.idx(x, y + 1 < d.ly ? y + 1 : 0, z),
                          d.idx(x, y, z + 1 < d.lz ? z + 1 : 0)};
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (q[j] != k && cls[q[j]] == c) uf_unite(parent, (int)k, (int)q[j]);
}

// Flatten every node onto its root and count the members of every root.
__global__ void k_flatten(const uint8_t* __restrict__ cls, Dims d,
                          int* __restrict__ parent, int* __restrict__ size) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  if (!cls[k]) return;
  const int r = uf_find(parent, (int)k);
  parent[k] = r;
  atomicAdd(size + r, 1);
}

// keep[k] = 1 for a root of a cluster of class c with >= kMinCluster nodes.
__global__ void k_keep(const uint8_t* __restrict__ cls, Dims d,
                       const int* __restrict__ parent,
                       const int* __restrict__ size, uint8_t c,
                       int* __restrict__ keep) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  keep[k] = (cls[k] == c && parent[k] == (int)k && size[k] >= kMinCluster) ? 1 : 0;
}

// Cluster number of every node of class c (0: not in a kept cluster);
// number = exclusive prefix of keep at the root + 1.
__global__ void k_number(const uint8_t* __restrict__ cls, Dims d,
                         const int* __restrict__ parent,
                         const int* __restrict__ keep,
                         const int* __restrict__ prefix, uint8_t c,
                         int* __restrict__ label) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  int v = 0;
  if (cls[k] == c) {
    const int r = parent[k];
    if (keep[r]) v = prefix[r] + 1;
  }
  label[k] = v;
}

// Liquid-solid / liquid-vapour boundary nodes: for a liquid node, the first
// neighbour x - e_i (i = 1..18) that is solid or not liquid decides.
__global__ void k_boundary(const uint8_t* __restrict__ fluid,
                           const float* __restrict__ rho,
                           const uint8_t* __restrict__ cls, Dims d, float rhol,
                           unsigned long long* __restrict__ counts) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n || cls[k] != 1) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  for (int i = 1; i < 19; ++i) {
    const int nx = (x - c_ex[i] + d.lx) % d.lx, ny = (y - c_ey[i] + d.ly) % d.ly,
              nz = (z - c_ez[i] + d.lz) % d.lz;
    const long long q = d.idx(nx, ny, nz);
    if (!fluid[q]) { atomicAdd(counts, 1ull); return; }
    if (rho[q] < rhol) { atomicAdd(counts + 1, 1ull); return; }
  }
}

// (liquid cluster number << 32 | solid number) of every 6-neighbour with a
// solid number of a node of a kept liquid cluster; n_keys counts them.
template <bool EMIT>
__global__ void k_solid_pairs(const int* __restrict__ label,
                              const int64_t* __restrict__ solid_number, Dims d,
                              unsigned long long* __restrict__ keys,
                              unsigned long long* __restrict__ n_keys) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  const int L = label[k];
  if (!L) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  const long long q[6] = {d.idx(x > 0 ? x - 1 : d.lx - 1, y, z),
                          d.idx(x, y > 0 ? y - 1 : d.ly - 1, z),
                          d.idx(x, y, z > 0 ? z - 1 : d.lz - 1),
                          d.idx(x < d.lx - 1 ? x + 1 : 0, y, z),
                          d.idx(x, y < d.ly - 1 ? y + 1 : 0, z),
                          d.idx(x, y, z < d.lz - 1 ? z + 1 : 0)};
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int64_t sn = solid_number[q[j]];
    if (sn == 0 || label[q[j]] == L) continue;
    const unsigned long long slot = atomicAdd(n_keys, 1ull);
    if (EMIT)
      keys[slot] = ((unsigned long long)(unsigned)L << 32) | (unsigned)(uint32_t)sn;
  }
}

// Distinct pairs and distinct clusters among sorted keys.
__global__ void k_count_distinct(const unsigned long long* __restrict__ keys,
                                 long long m,
                                 unsigned long long* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i == 0 || keys[i] != keys[i - 1]) atomicAdd(out, 1ull);
  if (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32)) atomicAdd(out + 1, 1ull);
}

// Single-cluster radius, part 1: does the cluster touch both faces of each
// axis (bits 0..2 of flags), and which x / y / z planes hold it (occ[0..lx),
// occ[lx..lx+ly), occ[lx+ly..lx+ly+lz)).
__global__ void k_faces(const int* __restrict__ label, Dims d,
                        unsigned* __restrict__ flags, int* __restrict__ occ) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n || label[k] != 1) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  occ[x] = 1;
  occ[d.lx + y] = 1;
  occ[d.lx + d.ly + z] = 1;
  if (x == 0 && label[d.idx(d.lx - 1, y, z)] == 1) atomicOr(flags, 1u);
  if (y == 0 && label[d.idx(x, d.ly - 1, z)] == 1) atomicOr(flags, 2u);
  if (z == 0 && label[d.idx(x, y, d.lz - 1)] == 1) atomicOr(flags, 4u);
}

// Nodes of class c.
__global__ void k_count_class(const uint8_t* __restrict__ cls, long long n,
                              uint8_t c, unsigned long long* __restrict__ out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool hit = k < n && cls[k] == c;
  const unsigned ballot = __ballot_sync(0xffffffffu, hit);
  if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(out, (unsigned long long)__popc(ballot));
}

struct Unwrap {
  bool xb, yb, zb;
  int xv, yv, zv;
};

// part 2: unwrapped coordinate sums and the node count
__global__ void k_centre_sums(const int* __restrict__ label, Dims d, Unwrap u,
                              unsigned long long* __restrict__ sums) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n || label[k] != 1) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  atomicAdd(sums, (unsigned long long)((u.xb && x < u.xv) ? x + d.lx : x));
  atomicAdd(sums + 1, (unsigned long long)((u.yb && y < u.yv) ? y + d.ly : y));
  atomicAdd(sums + 2, (unsigned long long)((u.zb && z < u.zv) ? z + d.lz : z));
  atomicAdd(sums + 3, 1ull);
}

// part 3: largest distance from the centre (float, each operation rounded on
// its own; sqrt in double as the host code); r >= 0, so the float bits order
// like the values
__global__ void k_radius(const int* __restrict__ label, Dims d, Unwrap u,
                         float xc, float yc, float zc,
                         unsigned* __restrict__ rmax_bits) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n || label[k] != 1) return;
  int x, y, z;
  d.xyz(k, x, y, z);
  const float ax = (float)((u.xb && x < u.xv) ? x + d.lx : x);
  const float ay = (float)((u.yb && y < u.yv) ? y + d.ly : y);
  const float az = (float)((u.zb && z < u.zv) ? z + d.lz : z);
  const float dxx = __fmul_rn(__fsub_rn(xc, ax), __fsub_rn(xc, ax));
  const float dyy = __fmul_rn(__fsub_rn(yc, ay), __fsub_rn(yc, ay));
  const float dzz = __fmul_rn(__fsub_rn(zc, az), __fsub_rn(zc, az));
  const float r2 = __fadd_rn(__fadd_rn(dxx, dyy), dzz);
  const float r = (float)sqrt((double)r2);
  atomicMax(rmax_bits, __float_as_uint(r));
}

}  // namespace
}  // namespace mlbm

namespace mlbm {
namespace {

mlbm_status cl_fail(cudaError_t e, const char* where) {
  cudaGetLastError();
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
  return set_error(MLBM_ERR_CUDA, msg);
}

// Device buffers of one call, freed on every return path.
struct ClBuffers {
  std::vector<void*> ptrs;
  ~ClBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t count) {
    void* v = nullptr;
    const cudaError_t e = cudaMalloc(&v, count * sizeof(T) + 16);
    if (e == cudaSuccess) ptrs.push_back(v);
    *p = static_cast<T*>(v);
    return e;
  }
};

#define CL_TRY(expr, where)                                \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return cl_fail(_e, where);      \
  } while (0)

}  // namespace
}  // namespace mlbm

using namespace mlbm;

extern "C" mlbm_status mlbm_cluster_stats_gpu(
    const float* rho, const uint8_t* is_fluid, const int64_t* solid_number,
    int32_t lx, int32_t ly, int32_t lz, float rhol, float rhog,
    int64_t solid_count, int32_t device, int64_t* liq_labels_out,
    int64_t* gas_labels_out, mlbm_stats_row* out) {
  if (!rho || !is_fluid || !out || lx < 1 || ly < 1 || lz < 1)
    return set_error(MLBM_ERR_ARG, "cluster_stats_gpu: bad arguments");
  const long long n = (long long)lx * ly * lz;
  if (n >= (1LL << 31))
    return set_error(MLBM_ERR_ARG, "cluster_stats_gpu: more than 2^31 nodes");
  mlbm::DeviceGuard restore_device;
  CL_TRY(cudaSetDevice(device), "cluster_stats_gpu");
  const Dims d{lx, ly, lz, n};
  const unsigned grid = (unsigned)((n + 255) / 256);
  ClBuffers b;
  float* d_rho;
  uint8_t *d_fluid, *d_cls;
  int64_t* d_sn = nullptr;
  int *d_parent, *d_size, *d_keep, *d_prefix, *d_liq, *d_gas;
  unsigned long long* d_cnt;  // [0,1] boundary, [2] keys, [3,4] distinct,
                              // [5..8] sums, [9] liquid nodes
  unsigned* d_flags;          // [0] faces, [1] max radius bits
  int* d_occ;
  CL_TRY(b.alloc(&d_rho, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_fluid, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_cls, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_parent, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_size, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_keep, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_prefix, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_liq, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_gas, n), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_cnt, 16), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_flags, 4), "cluster_stats_gpu buffers");
  CL_TRY(b.alloc(&d_occ, (size_t)lx + ly + lz), "cluster_stats_gpu buffers");
  CL_TRY(cudaMemcpy(d_rho, rho, n * sizeof(float), cudaMemcpyHostToDevice),
         "cluster_stats_gpu upload");
  CL_TRY(cudaMemcpy(d_fluid, is_fluid, n, cudaMemcpyHostToDevice),
         "cluster_stats_gpu upload");
  if (solid_number) {
    CL_TRY(b.alloc(&d_sn, n), "cluster_stats_gpu buffers");
    CL_TRY(cudaMemcpy(d_sn, solid_number, n * sizeof(int64_t), cudaMemcpyHostToDevice),
           "cluster_stats_gpu upload");
  }
  CL_TRY(cudaMemset(d_size, 0, n * sizeof(int)), "cluster_stats_gpu");
  CL_TRY(cudaMemset(d_cnt, 0, 16 * sizeof(unsigned long long)), "cluster_stats_gpu");
  CL_TRY(cudaMemset(d_flags, 0, 4 * sizeof(unsigned)), "cluster_stats_gpu");
  CL_TRY(cudaMemset(d_occ, 0, ((size_t)lx + ly + lz) * sizeof(int)), "cluster_stats_gpu");

  // components of both classes, each rooted at its first node in the scan
  k_classify<<<grid, 256>>>(d_rho, d_fluid, d, rhol, rhog, d_cls, d_parent);
  k_unite<<<grid, 256>>>(d_cls, d, d_parent);
  k_flatten<<<grid, 256>>>(d_cls, d, d_parent, d_size);
  CL_TRY(cudaGetLastError(), "cluster_stats_gpu labelling");

  // cluster numbers of the kept clusters, per class
  size_t scan_bytes = 0;
  CL_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_keep, d_prefix, (int)n),
         "cluster_stats_gpu scan");
  void* d_scan;
  CL_TRY(b.alloc(reinterpret_cast<unsigned char**>(&d_scan), scan_bytes),
         "cluster_stats_gpu buffers");
  long long counts[2] = {0, 0};
  for (int c = 1; c <= 2; ++c) {
    int* lab = c == 1 ? d_liq : d_gas;
    k_keep<<<grid, 256>>>(d_cls, d, d_parent, d_size, (uint8_t)c, d_keep);
    CL_TRY(cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_keep, d_prefix, (int)n),
           "cluster_stats_gpu scan");
    k_number<<<grid, 256>>>(d_cls, d, d_parent, d_keep, d_prefix, (uint8_t)c, lab);
    int last_p = 0, last_k = 0;
    CL_TRY(cudaMemcpy(&last_p, d_prefix + n - 1, sizeof(int), cudaMemcpyDeviceToHost),
           "cluster_stats_gpu count");
    CL_TRY(cudaMemcpy(&last_k, d_keep + n - 1, sizeof(int), cudaMemcpyDeviceToHost),
           "cluster_stats_gpu count");
    counts[c - 1] = (long long)last_p + last_k;
  }
  const long long liq_count = counts[0], gas_count = counts[1];

  // boundary ratios over all liquid nodes (kept clusters or not), :278-316
  k_boundary<<<grid, 256>>>(d_fluid, d_rho, d_cls, d, rhol, d_cnt);
  k_count_class<<<grid, 256>>>(d_cls, n, 1, d_cnt + 9);
  unsigned long long h_cnt[10];
  CL_TRY(cudaMemcpy(h_cnt, d_cnt, sizeof h_cnt, cudaMemcpyDeviceToHost),
         "cluster_stats_gpu boundary");
  const long long liquid_nodes = (long long)h_cnt[9];
  if (liquid_nodes > 0) {
    out->liquid_solid_boundary = (float)((double)h_cnt[0] / liquid_nodes);
    out->liquid_vapor_boundary = (float)((double)h_cnt[1] / liquid_nodes);
  }
  out->liq_cluster_count = liq_count;
  out->gas_cluster_count = gas_count;

  // cluster order and wet coordination number from the distinct
  // (liquid cluster, solid number) pairs, :535-561
  unsigned long long pairs = 0, touching = 0;
  if (d_sn && liq_count > 0) {
    k_solid_pairs<false><<<grid, 256>>>(d_liq, d_sn, d, nullptr, d_cnt + 2);
    unsigned long long m = 0;
    CL_TRY(cudaMemcpy(&m, d_cnt + 2, sizeof m, cudaMemcpyDeviceToHost),
           "cluster_stats_gpu pairs");
    if (m >= (1ull << 31))
      return set_error(MLBM_ERR_ARG, "cluster_stats_gpu: too many cluster-solid contacts");
    if (m > 0) {
      unsigned long long *d_keys, *d_sorted;
      CL_TRY(b.alloc(&d_keys, m), "cluster_stats_gpu pairs");
      CL_TRY(b.alloc(&d_sorted, m), "cluster_stats_gpu pairs");
      CL_TRY(cudaMemset(d_cnt + 2, 0, sizeof(unsigned long long)), "cluster_stats_gpu");
      k_solid_pairs<true><<<grid, 256>>>(d_liq, d_sn, d, d_keys, d_cnt + 2);
      size_t sort_bytes = 0;
      CL_TRY(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, d_keys, d_sorted,
                                            (int)m),
             "cluster_stats_gpu sort");
      unsigned char* d_sort;
      CL_TRY(b.alloc(&d_sort, sort_bytes), "cluster_stats_gpu sort");
      CL_TRY(cub::DeviceRadixSort::SortKeys(d_sort, sort_bytes, d_keys, d_sorted,
                                            (int)m),
             "cluster_stats_gpu sort");
      k_count_distinct<<<(unsigned)((m + 255) / 256), 256>>>(d_sorted, (long long)m,
                                                             d_cnt + 3);
      unsigned long long dc[2];
      CL_TRY(cudaMemcpy(dc, d_cnt + 3, sizeof dc, cudaMemcpyDeviceToHost),
             "cluster_stats_gpu pairs");
      pairs = dc[0];
      touching = dc[1];
    }
  }
  // the reference sums per-cluster set sizes in float (integers, exact)
  float order = (float)pairs;
  if (liq_count != 0) order /= (float)touching;  // 0/0 = NaN when none touches
  out->cluster_order = order;
  float wet = (float)pairs;
  if (solid_count != 0) wet /= (float)solid_count;
  out->wet_coord_num = wet;

  // single liquid cluster: centre and radius with periodic unwrapping
  float max_r = 0.f;
  if (liq_count == 1) {
    k_faces<<<grid, 256>>>(d_liq, d, d_flags, d_occ);
    unsigned flags = 0;
    std::vector<int> occ((size_t)lx + ly + lz);
    CL_TRY(cudaMemcpy(&flags, d_flags, sizeof flags, cudaMemcpyDeviceToHost),
           "cluster_stats_gpu radius");
    CL_TRY(cudaMemcpy(occ.data(), d_occ, occ.size() * sizeof(int),
                      cudaMemcpyDeviceToHost),
           "cluster_stats_gpu radius");
    Unwrap u{(flags & 1u) != 0, (flags & 2u) != 0, (flags & 4u) != 0, 0, 0, 0};
    auto first_free = [&](int off, int len) {
      for (int i = 0; i < len; ++i)
        if (!occ[off + i]) return i;
      return 0;
    };
    if (u.xb) u.xv = first_free(0, lx);
    if (u.yb) u.yv = first_free(lx, ly);
    if (u.zb) u.zv = first_free(lx + ly, lz);
    k_centre_sums<<<grid, 256>>>(d_liq, d, u, d_cnt + 5);
    unsigned long long sums[4];
    CL_TRY(cudaMemcpy(sums, d_cnt + 5, sizeof sums, cudaMemcpyDeviceToHost),
           "cluster_stats_gpu radius");
    // integer division, as the reference (:496-498)
    const float xc = (float)(sums[0] / sums[3]), yc = (float)(sums[1] / sums[3]),
                zc = (float)(sums[2] / sums[3]);
    k_radius<<<grid, 256>>>(d_liq, d, u, xc, yc, zc, d_flags + 1);
    unsigned rbits = 0;
    CL_TRY(cudaMemcpy(&rbits, d_flags + 1, sizeof rbits, cudaMemcpyDeviceToHost),
           "cluster_stats_gpu radius");
    std::memcpy(&max_r, &rbits, sizeof max_r);
  }
  out->cluster_radius = max_r;

  // cluster numbers in the reference layout, when asked for
  for (int c = 0; c < 2; ++c) {
    int64_t* dst = c == 0 ? liq_labels_out : gas_labels_out;
    if (!dst) continue;
    std::vector<int> h((size_t)n);
    CL_TRY(cudaMemcpy(h.data(), c == 0 ? d_liq : d_gas, n * sizeof(int),
                      cudaMemcpyDeviceToHost),
           "cluster_stats_gpu labels");
    for (long long k = 0; k < n; ++k) dst[k] = h[k];
  }
  CL_TRY(cudaGetLastError(), "cluster_stats_gpu");
  return MLBM_OK;
}
