// compact2.cuh -- the two-pass time step over the compact (fluid-only)
// population layout of compact.cuh.
//
// Same passes as kernels.cuh / update_tma.cuh (density pass: rho and psi of
// every fluid node; update pass: force, velocity shift, BGK, AA store), with
// the populations addressed by compact index, so DRAM moves only fluid nodes'
// populations.  The local AA step runs one thread per pair of consecutive
// fluid nodes (pair.cuh: packed FP32 arithmetic, 8-byte accesses), the
// gather/push step one thread per node; consecutive threads hold
// x-consecutive fluid nodes of a row, so
// own-slot accesses are coalesced and neighbour-slot accesses (phase 0) fall
// in the neighbouring rows' compact ranges.  No shared memory and no
// barriers.  Results are bit-identical to the dense two-pass kernels (same
// loads, same arithmetic in the same order).
//
// Per fluid node k: cinfo[k] = (neighbour word, packed coordinates
// x | y << 11 | z << 22); psi is the dense ghost-padded array of lattice.cuh,
// so psi of the 18 neighbours sits at fixed offsets from psi_index(x, y, z).
// `inj` is the injection step test of the launch (the same for every node).
#pragma once

#include "compact.cuh"
#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

constexpr int kC2Threads = 256;

__host__ __device__ constexpr uint32_t pack_xyz(int x, int y, int z) {
  return (uint32_t)x | ((uint32_t)y << 11) | ((uint32_t)z << 22);
}
// Largest edges the packed coordinates hold.
constexpr int kC2MaxX = 2048, kC2MaxY = 2048, kC2MaxZ = 1024;

// Neighbour words and packed coordinates of the fluid nodes, compact order.
static __global__ void k_cinfo(const uint32_t* __restrict__ nbw,
                               uint2* __restrict__ cinfo, CArgs c, Geom g) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(c.mask, g, x, y, z)) return;
  const long long k = compact_index(c, g, x, y, z);
  cinfo[k] = make_uint2(nbw[node_index(g, x, y, z)], pack_xyz(x, y, z));
}

// Compact indices of the 18 neighbours x + e_i of fluid node k at (x, y, z)
// (meaningful where the neighbour is fluid): the rank of x in each
// neighbour row from wtab[word] = (mask word, wbase), then x - 1 -> rank - 1
// and x + 1 -> rank + fluid(x), with the periodic wrap in x (row start =
// wtab[first word].y; the last node of a row = wtab[last word].y +
// popc(last word) - 1).  32-bit indices: the table has fewer than 2^31
// words.
__device__ __forceinline__ void neighbour_ranks(const uint2* __restrict__ wtab,
                                                const Geom& g, int k, int x,
                                                int y, int z, int (&nk)[Q]) {
  const int ym = y == 0 ? g.ly - 1 : y - 1, yp = y == g.ly - 1 ? 0 : y + 1;
  const int zm = z == 0 ? g.lz - 1 : z - 1, zp = z == g.lz - 1 ? 0 : z + 1;
  const bool xlo = x == 0, xhi = x == g.lx - 1;
  const int w = x >> 5, xb = x & 31;
  const uint32_t lb = low_bits(x);
  const int wpr = g.wpr;
  const int pz = z * g.ly, pzm = zm * g.ly, pzp = zp * g.ly;
  auto row_last = [&](int rb) {  // compact index of the row's last node
    const uint2 e = __ldg(wtab + rb + wpr - 1);
    return (int)e.y + __popc(e.x) - 1;
  };
  auto rank3 = [&](int row, int& r_, int& rl, int& rh) {
    const int rb = row * wpr;
    const uint2 v = __ldg(wtab + rb + w);
    r_ = (int)v.y + __popc(v.x & lb);
    rl = xlo ? row_last(rb) : r_ - 1;
    rh = xhi ? (int)__ldg(wtab + rb).y : r_ + (int)((v.x >> xb) & 1u);
  };
  auto rank1 = [&](int row) {
    const uint2 v = __ldg(wtab + row * wpr + w);
    return (int)v.y + __popc(v.x & lb);
  };
  const int r0 = (pz + y) * wpr;
  nk[0] = k;
  nk[1] = xlo ? row_last(r0) : k - 1;                        // (-1, 0, 0)
  nk[10] = xhi ? (int)__ldg(wtab + r0).y : k + 1;           // (+1, 0, 0)
  int r_, rl, rh;
  rank3(pz + ym, r_, rl, rh);  nk[2] = r_;  nk[4] = rl; nk[14] = rh;
  rank3(pz + yp, r_, rl, rh);  nk[11] = r_; nk[5] = rl; nk[13] = rh;
  rank3(pzm + y, r_, rl, rh);  nk[3] = r_;  nk[6] = rl; nk[16] = rh;
  rank3(pzp + y, r_, rl, rh);  nk[12] = r_; nk[7] = rl; nk[15] = rh;
  nk[8] = rank1(pzm + ym);   // (0, -1, -1)
  nk[9] = rank1(pzp + ym);   // (0, -1, +1)
  nk[17] = rank1(pzp + yp);  // (0, +1, +1)
  nk[18] = rank1(pzm + yp);  // (0, +1, -1)
}

// wtab[i] = (mask word i, wbase[i]); wtab[nwords] = (0, fluid node count).
static __global__ void k_wtab(const uint32_t* __restrict__ mask,
                              const uint32_t* __restrict__ wbase,
                              uint2* __restrict__ wtab, long long nwords) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= nwords) wtab[i] = make_uint2(i < nwords ? mask[i] : 0u, wbase[i]);
}

}  // namespace mlbm

#include "pair.cuh"

namespace mlbm {

// The update pass runs one thread per pair of fluid nodes (pair.cuh, k = 2 *
// thread index) in both AA phases; the gather/push form (phase 0) keeps its
// addresses in shared memory across the collision.  The density pass runs
// pairs in the local phase and one node per thread in the gather phase
// (pairs there measured 1 % slower at 64 and at 80 registers).
// The density pass is held to 48 registers (5 CTAs per SM); on the 200^3
// bench that beat 3, 4 and 6 CTAs per SM.  Both kernels advance the compact
// indices [kbeg, nfluid): the whole lattice, or the own planes of a slab
// lattice (kbeg is a plane start, so it is even).
template <int PHASE>
constexpr int c2_nodes_per_thread() { return PHASE == 0 ? 1 : 2; }
constexpr int c2_update_nodes_per_thread() { return 2; }

// Both kernels pass pdl_gate() (pair.cuh): launched with programmatic
// stream serialization, each overlaps its prologue with the end of the
// kernel before it.
template <typename T, int PHASE, bool WRITE_RHO>
__global__ void __launch_bounds__(kC2Threads, 5)
    k_cdensity(const T* __restrict__ cpop, uint32_t cs,
               const uint2* __restrict__ cinfo, const uint2* __restrict__ wtab,
               int kbeg, int nfluid, float* __restrict__ rho_out,
               float* __restrict__ psi, Geom g, Phys p, StepArgs a, bool inj) {
  const long long k = kbeg + c2_nodes_per_thread<PHASE>() *
                                 ((long long)blockIdx.x * kC2Threads + threadIdx.x);
  if (k >= nfluid) return;
  if (PHASE == 0)
    node_density0<T, WRITE_RHO, true>(cpop, cs, cinfo, wtab, (int)k, rho_out,
                                      psi, g, p, a, inj);
  else
    pair_density<T, 1, WRITE_RHO, true>(cpop, cs, cinfo, wtab, (int)k, nfluid,
                                        rho_out, psi, g, p, a, inj);
}

template <typename T, int PHASE, bool WRITE_U>
__global__ void __launch_bounds__(kC2Threads, 3)
    k_cupdate(T* __restrict__ cpop, uint32_t cs, const uint2* __restrict__ cinfo,
              const uint2* __restrict__ wtab, int kbeg, int nfluid,
              const float* __restrict__ psi, float* __restrict__ vel, Geom g,
              Phys p, StepArgs a, bool inj) {
  const long long k = kbeg + c2_update_nodes_per_thread() *
                                 ((long long)blockIdx.x * kC2Threads + threadIdx.x);
  if (k >= nfluid) return;
  pair_update<T, PHASE, WRITE_U, PsiPlain, true>(cpop, cs, cinfo, wtab, (int)k,
                                                 nfluid, PsiPlain{psi}, vel, g,
                                                 p, a, inj);
}

}  // namespace mlbm
