// compact.cuh -- the fluid-only ("compact") population layout.
//
// Fluid nodes are numbered in (z, y, x) order; population i of the fluid
// node numbered k lives at cpop[i * cs + k].  Solid nodes own no storage, so
// DRAM moves 19 reads and 19 writes per fluid node and nothing for solids.
// The index of a fluid node is found from the one-bit-per-node mask:
// wbase[r * wpr + w] is the compact index of the first fluid node at or
// after word w of row r = z * ly + y, so k(x, y, z) = wbase[r * wpr +
// x / 32] + popc(mask word & bits below x).  A plane with an odd fluid count
// is followed by one unused slot (a hole), so every plane starts at an even
// index; the end of row r is therefore wbase + popc of its last word (not
// always the next row's start).  wbase has one extra entry at the end (the
// slot count).  cnb[k] is the neighbour word of node k (kernels.cuh: bit 0
// fluid, bit i the pull source x - e_i fluid, bits 19-20 the drainage slab
// kind).
//
// The AA pattern and the slot conventions are those of kernels.cuh, with the
// compact index in place of the dense node index.  The step kernels over
// this layout are in compact2.cuh / pair.cuh (two passes) and band.cuh (one
// pass).
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

// Tables of the compact layout (device pointers).
struct CArgs {
  const uint32_t* mask;   // [rows][wpr]
  const uint32_t* wbase;  // [rows * wpr + 1]
  long long cs;           // compact plane stride (elements)
};

__device__ __forceinline__ uint32_t low_bits(int x) {
  return (1u << (x & 31)) - 1u;
}

// Compact index of node (x, y, z) from the global tables (the node must be
// fluid).
__device__ __forceinline__ long long compact_index(const CArgs& c,
                                                   const Geom& g, int x, int y,
                                                   int z) {
  const long long r = (long long)z * g.ly + y;
  const uint32_t w = __ldg(c.mask + r * g.wpr + (x >> 5));
  return (long long)__ldg(c.wbase + r * g.wpr + (x >> 5)) +
         __popc(w & low_bits(x));
}

// Per-word fluid counts of every mask row (the host scans them into wbase).
static __global__ void k_word_counts(const uint32_t* __restrict__ mask,
                                     uint32_t* __restrict__ counts,
                                     long long nwords) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nwords) counts[i] = __popc(mask[i]);
}

// Dense <-> compact copies of the populations (all slots of fluid nodes).
template <typename T, bool TO_COMPACT>
__global__ void k_convert(T* __restrict__ dense, T* __restrict__ cpop,
                          CArgs c, Geom g) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(c.mask, g, x, y, z)) return;
  const long long n = node_index(g, x, y, z);
  const long long k = compact_index(c, g, x, y, z);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if (TO_COMPACT)
      cpop[i * c.cs + k] = dense[i * g.plane + n];
    else
      dense[i * g.plane + n] = cpop[i * c.cs + k];
  }
}

// The density injection of compute_density (include/iteration_device.cuh:
// 46-59) with its step test, the same for every node of a launch, hoisted
// out: `on` is that test.
__device__ __forceinline__ float inject_on(const Phys& p, const Geom& g,
                                           const StepArgs& s, bool on, int y,
                                           float d) {
  if (!on || !((float)y < p.inject_position * (float)g.ly)) return d;
  const float inc = rmul(p.rho_increment, (float)s.reverse);
  switch (s.inject_type) {
    case 0: return radd(d, inc);
    case 1: return d < p.rhol_spinodal ? radd(d, inc) : d;
    case 2: return d > p.rhol_spinodal ? radd(d, inc) : d;
    default: return d;
  }
}

}  // namespace mlbm
