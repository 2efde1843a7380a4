// compact2.cuh -- the two-pass time step over the compact (fluid-only)
// population layout of compact.cuh.
//
// Same passes as kernels.cuh / update_tma.cuh (density pass: rho and psi of
// every fluid node; update pass: force, velocity shift, BGK, AA store), with
// the populations addressed by compact index, so DRAM moves only fluid nodes'
// populations.  One thread per fluid node, in compact order: consecutive
// threads hold x-consecutive fluid nodes of a row, so own-slot accesses are
// coalesced and neighbour-slot accesses (phase 0) fall in the neighbouring
// rows' compact ranges.  No shared memory and no barriers: every warp keeps
// its 19 loads in flight independently.  Results are bit-identical to the
// dense two-pass kernels (same loads, same arithmetic in the same order).
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
// wtab[first word].y, row end = wtab[first word + wpr].y, the next row's
// start; wtab has one sentinel entry after the last row).  32-bit indices:
// the table has fewer than 2^31 words.
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
  auto rank3 = [&](int row, int& r_, int& rl, int& rh) {
    const int rb = row * wpr;
    const uint2 v = __ldg(wtab + rb + w);
    r_ = (int)v.y + __popc(v.x & lb);
    rl = xlo ? (int)__ldg(wtab + rb + wpr).y - 1 : r_ - 1;
    rh = xhi ? (int)__ldg(wtab + rb).y : r_ + (int)((v.x >> xb) & 1u);
  };
  auto rank1 = [&](int row) {
    const uint2 v = __ldg(wtab + row * wpr + w);
    return (int)v.y + __popc(v.x & lb);
  };
  const int r0 = (pz + y) * wpr;
  nk[0] = k;
  nk[1] = xlo ? (int)__ldg(wtab + r0 + wpr).y - 1 : k - 1;  // (-1, 0, 0)
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

template <typename T, int PHASE>
__device__ __forceinline__ void cgather(const T* __restrict__ cpop, long long cs,
                                        int k, uint32_t nb, const int (&nk)[Q],
                                        float shift, float (&f)[Q]) {
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const float s = shift * weight<float>(i);
    int src = k, slot = i;
    if (PHASE == 0 && i != 0 && ((nb >> i) & 1u)) {
      src = nk[opp(i)];
      slot = opp(i);
    }
    f[i] = Pop<T>::ld(cpop + slot * cs + src, s);
  }
}

template <typename T, int PHASE, bool WRITE_RHO>
__global__ void __launch_bounds__(kC2Threads)
    k_cdensity(const T* __restrict__ cpop, CArgs c,
               const uint2* __restrict__ cinfo, const uint2* __restrict__ wtab,
               long long nfluid,
               float* __restrict__ rho_out, float* __restrict__ psi, Geom g,
               Phys p, StepArgs a, bool inj) {
  const long long kk = (long long)blockIdx.x * kC2Threads + threadIdx.x;
  if (kk >= nfluid) return;
  const int k = (int)kk;
  const uint2 ci = cinfo[k];
  const uint32_t nb = ci.x;
  const int x = (int)(ci.y & 2047u), y = (int)((ci.y >> 11) & 2047u),
            z = (int)(ci.y >> 22);
  const int kind = nb_kind(nb);
  float d;
  if (kind) {
    d = slab_density(p, kind);
  } else {
    int nk[Q];
    if (PHASE == 0) neighbour_ranks(wtab, g, k, x, y, z, nk);
    float f[Q];
    cgather<T, PHASE>(cpop, c.cs, k, nb, nk, p.rho_shift, f);
    d = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
    d = inject_on(p, g, a, inj, y, d);
  }
  if (WRITE_RHO) rho_out[node_index(g, x, y, z)] = d;
  store_psi<float>(psi, g, x, y, z, psi_of<float>(p, d));
}

template <typename T, int PHASE, bool WRITE_U>
__global__ void __launch_bounds__(kC2Threads)
    k_cupdate(T* __restrict__ cpop, CArgs c, const uint2* __restrict__ cinfo,
              const uint2* __restrict__ wtab, long long nfluid,
              const float* __restrict__ psi,
              float* __restrict__ vel, Geom g, Phys p, StepArgs a, bool inj) {
  const long long kk = (long long)blockIdx.x * kC2Threads + threadIdx.x;
  if (kk >= nfluid) return;
  const int k = (int)kk;
  const uint2 ci = cinfo[k];
  const uint32_t nb = ci.x;
  const int x = (int)(ci.y & 2047u), y = (int)((ci.y >> 11) & 2047u),
            z = (int)(ci.y >> 22);
  const int kind = nb_kind(nb);
  const float shift = p.rho_shift;
  int nk[Q];
  if (PHASE == 0) neighbour_ranks(wtab, g, k, x, y, z, nk);
  float f[Q];
  float ux = 0.f, uy = 0.f, uz = 0.f;
  if (kind) {
    slab_populations<float>(slab_density(p, kind), f);
  } else {
    cgather<T, PHASE>(cpop, c.cs, k, nb, nk, shift, f);
    float d = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
    d = inject_on(p, g, a, inj, y, d);
    const long long pc = psi_index(g, x, y, z);
    const long long sy = g.pxg, sz = (long long)(g.ly + 2) * g.pxg;
    collide<float>(
        p, d, __ldg(psi + pc),
        [&](int i) { return __ldg(psi + pc + ex(i) + ey(i) * sy + ez(i) * sz); },
        f, ux, uy, uz);
  }
  if (WRITE_U) {
    const long long n = node_index(g, x, y, z);
    vel[3 * n] = ux;
    vel[3 * n + 1] = uy;
    vel[3 * n + 2] = uz;
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const float s = shift * weight<float>(i);
    int dst = k, slot = opp(i);
    if (PHASE == 0 && i != 0 && ((nb >> opp(i)) & 1u)) {
      dst = nk[i];
      slot = i;
    }
    Pop<T>::st(cpop + slot * c.cs + dst, f[i], s);
  }
}

}  // namespace mlbm
