// io_kernels.cuh -- layout conversion between the reference's [x][y][z]
// arrays and the internal structure-of-arrays lattice, and the device
// reductions behind the phase statistics.
#pragma once

#include "lattice.cuh"

namespace mlbm {

// Reference layout index: ((x * ly + y) * lz + z), z fastest
// (include/lbm_model.cuh:18-22).
__device__ __forceinline__ long long ref_index(const Geom& g, int x, int y,
                                               int z) {
  return ((long long)x * g.ly + y) * g.lz + z;
}

// Internal-layout kernels use blockDim (32, 4) over (x, y) and grid.z = z.
#define MLBM_NODE_COORDS                              \
  const int x = blockIdx.x * 32 + threadIdx.x;        \
  const int y = blockIdx.y * blockDim.y + threadIdx.y; \
  const int z = blockIdx.z;

// Pack a uint8 [x][y][z] fluid array into the bit mask; every warp covers one
// aligned 32-node run of a row.
__global__ void k_pack_mask(const uint8_t* __restrict__ fluid_ref,
                            uint32_t* __restrict__ mask, Geom g) {
  MLBM_NODE_COORDS
  if (y >= g.ly) return;  // whole warp exits together (warp = one row run)
  const bool f = (x < g.lx) && fluid_ref[ref_index(g, x, y, z)] != 0;
  const uint32_t w = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0)
    mask[((long long)z * g.ly + y) * g.wpr + (x >> 5)] = w;
}

__global__ void k_rho_from_ref(const float* __restrict__ rho_ref,
                               float* __restrict__ rho_int, Geom g) {
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  rho_int[node_index(g, x, y, z)] = rho_ref[ref_index(g, x, y, z)];
}

// field: 0 rho, 1 pressure, 2 psi, 5 fluid (as 0/1) -> reference layout.
template <typename R, typename O>
__global__ void k_scalar_to_ref(const R* __restrict__ rho,
                                const uint32_t* __restrict__ mask,
                                O* __restrict__ out, Geom g, Phys p,
                                int field) {
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  const R r = rho[node_index(g, x, y, z)];
  R v;
  if (field == 0) v = r;
  else if (field == 1) v = pressure_of<R>(p, r);
  else if (field == 2) v = psi_of<R>(p, r);
  else v = R(fluid_at(mask, g, x, y, z) ? 1 : 0);
  out[ref_index(g, x, y, z)] = (O)v;
}

__global__ void k_fluid_to_ref(const uint32_t* __restrict__ mask,
                               uint8_t* __restrict__ out, Geom g) {
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  out[ref_index(g, x, y, z)] = fluid_at(mask, g, x, y, z) ? 1 : 0;
}

template <typename O>
__global__ void k_vel_to_ref(const float* __restrict__ vel,
                             O* __restrict__ out, Geom g) {
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  const long long n = node_index(g, x, y, z), r = ref_index(g, x, y, z);
  for (int c = 0; c < 3; ++c) out[3 * r + c] = (O)vel[3 * n + c];
}

// Post-collision populations f*_i in the reference layout [x][y][z][19].
// Phase 0: f*_i(x) = pop[opp(i)][x].  Phase 1 (fluid nodes): pop[i][x+e_i]
// when x+e_i is fluid, else pop[opp(i)][x].  Solid nodes keep their
// initial values, stored at pop[opp(i)][x] in either phase.
template <typename T, typename O>
__global__ void k_pop_to_ref(const T* __restrict__ pop,
                             const uint32_t* __restrict__ mask,
                             O* __restrict__ out, Geom g, Phys p, int phase) {
  using R = typename Pop<T>::Real;
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  const long long n = node_index(g, x, y, z), r = ref_index(g, x, y, z);
  const bool fl = fluid_at(mask, g, x, y, z);
  const R shift = R(p.rho_shift);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R s = shift * weight<R>(i);
    long long src = opp(i) * g.plane + n;
    if (phase == 1 && fl && i != 0) {
      const int xd = wrapc(x + ex(i), g.lx), yd = wrapc(y + ey(i), g.ly),
                zd = wrapc(z + ez(i), g.lz);
      if (fluid_at(mask, g, xd, yd, zd))
        src = i * g.plane + node_index(g, xd, yd, zd);
    }
    out[(long long)Q * r + i] = (O)Pop<T>::ld(pop + src, s);
  }
}

// ---- phase statistics ----------------------------------------------------------
// Per node of the fluid: counts (fluid, liquid, vapour, liquid-solid and
// liquid-vapour boundary nodes), FP64 sums (mass, liquid/vapour pressure and
// density) and min/max of rho and p.  calc_cluster, src/multiphase_lbm.cu:
// 240-316; write_stats, :1061-1072.
enum { ST_NF, ST_NL, ST_NV, ST_NLS, ST_NLV, ST_MASS, ST_PL, ST_PV, ST_RL,
       ST_RV, ST_MINR, ST_MAXR, ST_MINP, ST_MAXP, ST_COUNT };

constexpr int kStatThreads = 256;  // blockDim (32, 8)
constexpr int kStatZ = 16;         // planes per block

__device__ __forceinline__ double stat_op(int k, double v, double o) {
  return (k == ST_MINR || k == ST_MINP) ? fmin(v, o)
         : (k == ST_MAXR || k == ST_MAXP) ? fmax(v, o)
                                           : v + o;
}
__device__ __forceinline__ double stat_identity(int k) {
  return (k == ST_MINR || k == ST_MINP) ? 1e9
         : (k == ST_MAXR || k == ST_MAXP) ? -1e-9
                                           : 0.0;
}

// The statistics of one fluid node folded into acc.  The liquid boundary
// test reads the node's neighbour word (bit i: x - e_i is fluid) and the
// density of every fluid neighbour, then takes the first neighbour
// (i = 1..18) that is solid or not liquid, as calc_cluster does.  FULL =
// false folds only the bulk columns (stat_bulk_column): no boundary test and
// no pressure; those columns get the same operations in the same order
// either way, so they come out bit-identical.
template <typename R, bool FULL = true>
__device__ __forceinline__ void stat_node(double (&acc)[ST_COUNT],
                                          const R* __restrict__ rho,
                                          const Geom& g, const Phys& p, int x,
                                          int y, int z, uint32_t nb, R r) {
  const R rhol = R(p.rhol_spinodal), rhog = R(p.rhog_spinodal);
  const R pr = FULL ? pressure_of<R>(p, r) : R(0);
  acc[ST_NF] += 1.0;
  acc[ST_MASS] += (double)r;
  if (r > rhol) {
    acc[ST_NL] += 1.0;
    if (FULL) acc[ST_PL] += (double)pr;
    acc[ST_RL] += (double)r;
    if (FULL) {
      Nbr a;
      a.init(g, x, y, z);
      // all 18 neighbour densities as independent loads (every periodic
      // index lies inside the array, solid nodes included), then the masks:
      // a load under each direction's branch would wait on the one before
      R nr[Q];
#pragma unroll
      for (int i = 1; i < Q; ++i) nr[i] = __ldg(rho + a.idx(-ex(i), -ey(i), -ez(i)));
      const uint32_t solid = ~nb & 0x7fffeu;  // directions 1..18
      uint32_t low = 0u;
#pragma unroll
      for (int i = 1; i < Q; ++i) low |= (nr[i] < rhol ? 1u : 0u) << i;
      const uint32_t other = low & nb & 0x7fffeu;
      const uint32_t first = (solid | other) & (0u - (solid | other));
      if (first & solid) acc[ST_NLS] += 1.0;
      else if (first) acc[ST_NLV] += 1.0;
    }
  } else if (r < rhog) {
    acc[ST_NV] += 1.0;
    if (FULL) acc[ST_PV] += (double)pr;
    acc[ST_RV] += (double)r;
  }
  acc[ST_MINR] = fmin(acc[ST_MINR], (double)r);
  acc[ST_MAXR] = fmax(acc[ST_MAXR], (double)r);
  if (FULL) {
    acc[ST_MINP] = fmin(acc[ST_MINP], (double)pr);
    acc[ST_MAXP] = fmax(acc[ST_MAXP], (double)pr);
  }
}

// The columns that the bulk statistics (FULL = false) compute; the others
// are written as 0.
__host__ __device__ constexpr bool stat_bulk_column(int k) {
  return k == ST_NF || k == ST_NL || k == ST_NV || k == ST_MASS ||
         k == ST_RL || k == ST_RV || k == ST_MINR || k == ST_MAXR;
}

// Warp then block reduction of acc in a fixed order (deterministic); thread 0
// .. ST_COUNT - 1 of the block write the block's record.  256 threads.
__device__ __forceinline__ void stat_block_reduce(double (&acc)[ST_COUNT],
                                                  int tid, double* record) {
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) {
    double v = acc[k];
    for (int off = 16; off > 0; off >>= 1)
      v = stat_op(k, v, __shfl_down_sync(0xffffffffu, v, off));
    acc[k] = v;
  }
  __shared__ double sh[kStatThreads / 32][ST_COUNT];
  const int warp = tid >> 5, lane = tid & 31;
  if (lane == 0)
    for (int k = 0; k < ST_COUNT; ++k) sh[warp][k] = acc[k];
  __syncthreads();
  if (tid < ST_COUNT) {
    const int k = tid;
    double v = sh[0][k];
    for (int w = 1; w < kStatThreads / 32; ++w) v = stat_op(k, v, sh[w][k]);
    record[k] = v;
  }
}

// Scratch of one statistics reduction (8-byte slots): slot 0 the arrival
// counter (zero between calls), then the block records (ST_COUNT each),
// then the ST_COUNT results and the device error flag.
struct StatScratch {
  unsigned* counter;
  double* records;
  double* out;
};

// Called by every thread of a block once the block's record is written
// (stat_block_reduce).  The last block to arrive folds all records -- in a
// fixed order, so the result does not depend on which block is last: thread
// t folds records t, t + 256, ... ascending, then the warps' shuffle trees,
// then the warps in order -- writes the results and the device error flag
// and re-arms the counter.  Records are read through L2 (ld.global.cg):
// other SMs wrote them.  256 threads.
__device__ __forceinline__ void stat_last_block(StatScratch s, unsigned nblocks,
                                                const int* __restrict__ err,
                                                int tid, bool full) {
  __shared__ bool last;
  __shared__ double sh[kStatThreads / 32][ST_COUNT];
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(s.counter, 1u) == nblocks - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v[ST_COUNT];
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) v[k] = stat_identity(k);
  for (unsigned b = tid; b < nblocks; b += kStatThreads) {
    const double* rec = s.records + (size_t)b * ST_COUNT;
    double r[ST_COUNT];
#pragma unroll
    for (int k = 0; k < ST_COUNT; ++k) r[k] = __ldcg(rec + k);
#pragma unroll
    for (int k = 0; k < ST_COUNT; ++k) v[k] = stat_op(k, v[k], r[k]);
  }
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k)
    for (int off = 16; off > 0; off >>= 1)
      v[k] = stat_op(k, v[k], __shfl_down_sync(0xffffffffu, v[k], off));
  const int warp = tid >> 5, lane = tid & 31;
  if (lane == 0)
    for (int k = 0; k < ST_COUNT; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (tid < ST_COUNT) {
    double r = sh[0][tid];
    for (int w = 1; w < kStatThreads / 32; ++w) r = stat_op(tid, r, sh[w][tid]);
    s.out[tid] = full || stat_bulk_column(tid) ? r : 0.0;  // not computed: 0
  }
  if (tid == 0) {
    s.out[ST_COUNT] = err ? (double)*err : 0.0;
    *s.counter = 0u;
  }
}

// Dense form: one block per 32 x 8 nodes of an (x, y) plane and kStatZ
// planes; each thread folds its column of nodes, z ascending.
template <typename R, bool FULL = true>
__global__ void __launch_bounds__(kStatThreads)
    k_stats_partial(const R* __restrict__ rho, const uint32_t* __restrict__ nbw,
                    Geom g, Phys p, StatScratch sc, const int* __restrict__ err) {
  double acc[ST_COUNT];
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) acc[k] = stat_identity(k);
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z0 = blockIdx.z * kStatZ, z1 = min(z0 + kStatZ, g.lz);
  if (x < g.lx && y < g.ly) {
    // eight planes' node words and densities in flight at once (4: 1 %
    // slower end to end; 8 planes per block with more blocks: 5 % slower)
    constexpr int U = 8;
#pragma unroll 1
    for (int zb = z0; zb < z1; zb += U) {
      uint32_t nbv[U];
      R rv[U];
#pragma unroll
      for (int j = 0; j < U; ++j) {
        nbv[j] = 0u;
        rv[j] = R(0);
        if (zb + j < z1) {
          const long long n = node_index(g, x, y, zb + j);
          nbv[j] = __ldg(nbw + n);
          rv[j] = __ldg(rho + n);
        }
      }
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (nbv[j] & NB_SELF)
          stat_node<R, FULL>(acc, rho, g, p, x, y, zb + j, nbv[j], rv[j]);
    }
  }
  const long long blk =
      blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
  const int tid = threadIdx.y * 32 + threadIdx.x;
  stat_block_reduce(acc, tid, sc.records + blk * ST_COUNT);
  stat_last_block(sc, gridDim.x * gridDim.y * gridDim.z, err, tid, FULL);
}

// Fluid-list form, for a lattice held in the fluid-only layout: the threads
// walk the compact node table (node word, packed x, y, z), so no lane idles
// on a solid node.  The grid is one wave of resident blocks (the host sizes
// it); block b folds slots [b * span, (b + 1) * span) and thread t takes
// slots t, t + 256, ... of them, ascending -- a fixed assignment, so the
// sums do not depend on scheduling.
template <typename R, bool FULL = true>
__global__ void __launch_bounds__(kStatThreads)
    k_stats_fluid(const R* __restrict__ rho, const uint2* __restrict__ cinfo,
                  long long nslots, long long span, Geom g, Phys p,
                  StatScratch sc, const int* __restrict__ err) {
  double acc[ST_COUNT];
#pragma unroll
  for (int k = 0; k < ST_COUNT; ++k) acc[k] = stat_identity(k);
  const long long b0 = (long long)blockIdx.x * span;
  const long long end = min(b0 + span, nslots);
  constexpr int U = 8;
#pragma unroll 1
  for (long long k0 = b0 + threadIdx.x; k0 < end; k0 += (long long)U * kStatThreads) {
    uint2 ci[U];
    R rv[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const long long k = k0 + (long long)j * kStatThreads;
      ci[j] = k < end ? __ldg(cinfo + k) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int j = 0; j < U; ++j) {
      rv[j] = R(0);
      if (ci[j].x & NB_SELF)
        rv[j] = __ldg(rho + node_index(g, (int)(ci[j].y & 2047u),
                                       (int)((ci[j].y >> 11) & 2047u),
                                       (int)(ci[j].y >> 22)));
    }
#pragma unroll
    for (int j = 0; j < U; ++j)
      if (ci[j].x & NB_SELF)
        stat_node<R, FULL>(acc, rho, g, p, (int)(ci[j].y & 2047u),
                     (int)((ci[j].y >> 11) & 2047u), (int)(ci[j].y >> 22),
                     ci[j].x, rv[j]);
  }
  stat_block_reduce(acc, threadIdx.x, sc.records + (long long)blockIdx.x * ST_COUNT);
  stat_last_block(sc, gridDim.x, err, threadIdx.x, FULL);
}

// Per-x-plane fluid / liquid node counts (integer atomics: deterministic).
template <typename R>
__global__ void k_plane_profile(const R* __restrict__ rho,
                                const uint32_t* __restrict__ mask, Geom g,
                                Phys p, unsigned long long* __restrict__ nf,
                                unsigned long long* __restrict__ nl) {
  MLBM_NODE_COORDS
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(mask, g, x, y, z)) return;
  atomicAdd(nf + x, 1ull);
  if (rho[node_index(g, x, y, z)] > R(p.rhol_spinodal)) atomicAdd(nl + x, 1ull);
}

}  // namespace mlbm
