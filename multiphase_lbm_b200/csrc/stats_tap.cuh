// stats_tap.cuh -- the phase statistics of a step gathered by the step's own
// update pass (compact layout, either AA phase) instead of a separate pass
// over the density field.
//
// calc_cluster (src/multiphase_lbm.cu:240-316) needs per fluid node its
// density and pressure and, for a liquid node (rho > rhol), the first of its
// 18 neighbours x - e_i (i = 1..18 in order) that is solid or not liquid
// (rho < rhol).  The update pass already forms the node's density (the same
// sum, in the same order, that the density pass stored) and has just loaded
// psi of all 18 neighbours for the interaction force (so reading them again
// after the update hits the cache), and the test "neighbour not liquid" is
// read off psi as psi < T.  That equals rho < rhol for every
// neighbour exactly when T separates psi(r) of all float densities r < rhol
// from psi(r) of all others; k_psi_threshold checks that for the lattice's
// psi function over all 2^32 float bit patterns and yields T, and the host
// gathers the statistics this way only where the check holds (otherwise the
// separate pass, io_kernels.cuh, runs).
//
// Counts and min/max are exact and independent of order; the FP64 sums are
// folded in a fixed order (node, lane pair, warp tree, block, then the
// block records by k_stats_final_cols), so the result is deterministic, and
// equal to the separate pass's sums up to the rounding of another
// summation order.
#pragma once

#include <cstdint>

#include "lattice.cuh"
#include "stat_defs.cuh"

namespace mlbm {

// Statistics of the nodes one thread updated (at most two).
struct StatAcc {
  unsigned nf, nl, nv, nls, nlv;
  double mass, pl, pv, rl, rv;
  float minr, maxr, minp, maxp;
  __device__ __forceinline__ void clear() {
    nf = nl = nv = nls = nlv = 0u;
    mass = pl = pv = rl = rv = 0.0;
    minr = minp = __int_as_float(0x7f800000);   // +inf
    maxr = maxp = __int_as_float(0xff800000);   // -inf
  }
  // One fluid node of density r.  nb: its neighbour word (bit i: x - e_i is
  // fluid); low: bit i set where psi of x - e_i is below the threshold (only
  // read for a liquid node).  The classification of stat_node.
  __device__ __forceinline__ void add(const Phys& p, float r, uint32_t nb,
                                      uint32_t low) {
    const float pr = pressure_of<float>(p, r);
    nf += 1u;
    mass += (double)r;
    if (r > p.rhol_spinodal) {
      nl += 1u;
      pl += (double)pr;
      rl += (double)r;
      const uint32_t solid = ~nb & 0x7fffeu;
      const uint32_t other = low & nb & 0x7fffeu;
      const uint32_t first = (solid | other) & (0u - (solid | other));
      if (first & solid) nls += 1u;
      else if (first) nlv += 1u;
    } else if (r < p.rhog_spinodal) {
      nv += 1u;
      pv += (double)pr;
      rv += (double)r;
    }
    minr = fminf(minr, r);
    maxr = fmaxf(maxr, r);
    minp = fminf(minp, pr);
    maxp = fmaxf(maxp, pr);
  }
};

// The neighbour-psi test of one node: bit i set where psi of x - e_i is
// below T (psi_index layout; periodic images live in the halo).
__device__ __forceinline__ uint32_t stat_low_bits(const float* __restrict__ psi,
                                                  const Geom& g, int x, int y,
                                                  int z, float T) {
  const long long c = psi_index(g, x, y, z);
  const int sy = g.pxg, sz = (g.ly + 2) * g.pxg;
  uint32_t low = 0u;
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const float v = __ldg(psi + c - (ex(i) + ey(i) * sy + ez(i) * sz));
    low |= (v < T ? 1u : 0u) << i;
  }
  return low;
}

// Fold one fluid node whose update is done: its node-table entry
// (neighbour word, packed x, y, z) and density r; a liquid node reads the
// psi of its 18 neighbours for the boundary test.
__device__ __forceinline__ void stat_fold_node(StatAcc& acc, const Phys& p,
                                               const Geom& g,
                                               const float* __restrict__ psi,
                                               uint2 ci, float r, float T) {
  uint32_t low = 0u;
  if (r > p.rhol_spinodal)
    low = stat_low_bits(psi, g, (int)(ci.y & 2047u), (int)((ci.y >> 11) & 2047u),
                        (int)(ci.y >> 22), T);
  acc.add(p, r, ci.x, low);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v = fminf(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

// Fold the block's accumulators (fixed order: warp trees, then warps
// ascending) and write them as record `rec` of column-major partials:
// part[k * nblk + rec] for statistic k.  Every thread of the block must
// call it.
template <int THREADS>
__device__ __forceinline__ void stat_block_write(const StatAcc& a,
                                                 double* __restrict__ part,
                                                 unsigned nblk, unsigned rec) {
  constexpr int W = THREADS / 32;
  __shared__ double sh[ST_COUNT][W];
  double v[ST_COUNT];
  v[ST_NF] = (double)__reduce_add_sync(0xffffffffu, a.nf);
  v[ST_NL] = (double)__reduce_add_sync(0xffffffffu, a.nl);
  v[ST_NV] = (double)__reduce_add_sync(0xffffffffu, a.nv);
  v[ST_NLS] = (double)__reduce_add_sync(0xffffffffu, a.nls);
  v[ST_NLV] = (double)__reduce_add_sync(0xffffffffu, a.nlv);
  v[ST_MASS] = warp_sum(a.mass);
  v[ST_PL] = warp_sum(a.pl);
  v[ST_PV] = warp_sum(a.pv);
  v[ST_RL] = warp_sum(a.rl);
  v[ST_RV] = warp_sum(a.rv);
  v[ST_MINR] = (double)warp_min(a.minr);
  v[ST_MAXR] = (double)warp_max(a.maxr);
  v[ST_MINP] = (double)warp_min(a.minp);
  v[ST_MAXP] = (double)warp_max(a.maxp);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < ST_COUNT; ++k) sh[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < ST_COUNT) {
    const int k = threadIdx.x;
    double r = sh[k][0];
#pragma unroll
    for (int w = 1; w < W; ++w) r = stat_op(k, r, sh[k][w]);
    part[(size_t)k * nblk + rec] = r;
  }
}

// The reduction of the partials (k_stats_final_cols) and the threshold check
// (k_psi_threshold) are launched by the host code of the compact kernels.

}  // namespace mlbm
