// lattice.cuh -- D3Q19 model, storage formats and Shan-Chen physics shared by
// every kernel of the B200 implementation.
//
// Direction order, weights and velocities are the reference's
// (include/lbm_model.cuh:35-54) so that populations are interchangeable with
// the reference's collision_f / stream_f arrays.  opposite(i) is i+9 / i-9
// (include/lbm_model.cuh:24), with opposite(0) = 0.
#pragma once

#include <cuda_fp16.h>
#include <limits.h>
#include <stdint.h>

namespace mlbm {

constexpr int Q = 19;

__host__ __device__ constexpr int ex(int i) {
  return (i == 0 || i == 2 || i == 3 || i == 8 || i == 9 || i == 11 ||
          i == 12 || i == 17 || i == 18)
             ? 0
             : (i < 10 ? -1 : 1);
}
__host__ __device__ constexpr int ey(int i) {
  return (i == 2 || i == 4 || i == 8 || i == 9 || i == 14) ? -1
         : (i == 5 || i == 11 || i == 13 || i == 17 || i == 18) ? 1
                                                                : 0;
}
__host__ __device__ constexpr int ez(int i) {
  return (i == 3 || i == 6 || i == 8 || i == 16 || i == 18) ? -1
         : (i == 7 || i == 9 || i == 12 || i == 15 || i == 17) ? 1
                                                                : 0;
}
__host__ __device__ constexpr int opp(int i) {
  return i == 0 ? 0 : (i > 9 ? i - 9 : i + 9);
}
// Lattice weights t_i (= the Shan-Chen weights w_i, include/lbm_model.cuh:45)
template <typename R>
__host__ __device__ constexpr R weight(int i) {
  return i == 0 ? R(1.0 / 3.0)
                : ((i <= 3 || (i >= 10 && i <= 12)) ? R(1.0 / 18.0)
                                                    : R(1.0 / 36.0));
}

// ---- geometry of one lattice in HBM --------------------------------------
// Structure of arrays: population i of node (x,y,z) lives at
//   pop[i * plane + (z * ly + y) * px + x]
// with the row pitch px a multiple of 32 nodes (128 B in FP32) so that every
// warp-wide row access is sector aligned.  Scalars (rho) use the same node
// index.  The solid mask is one bit per node: word (z*ly + y)*wpr + x/32,
// bit x%32, 1 = fluid.
struct Geom {
  int lx, ly, lz;
  int px;        // row pitch in nodes (multiple of 32)
  int wpr;       // mask words per row = px / 32
  long long plane;  // nodes per population plane = lz * ly * px
  int pxg;       // psi row pitch (px + 8, see psi_index)
};

// psi is stored with one ghost layer on every side, so a tile plus its halo
// is one rectangular box of memory even at the periodic boundaries:
// psi(x, y, z) at ((z + 1) * (ly + 2) + y + 1) * pxg + x + 4 for x in
// [-1, lx], y in [-1, ly], z in [-1, lz].  x starts at column 4 so that every
// 32-aligned tile's halo box starts 16-byte aligned (a TMA requirement).
__host__ __device__ __forceinline__ long long psi_index(const Geom& g, int x,
                                                       int y, int z) {
  return ((long long)(z + 1) * (g.ly + 2) + (y + 1)) * g.pxg + x + 4;
}
__host__ __device__ __forceinline__ long long psi_elems(const Geom& g) {
  return (long long)(g.lz + 2) * (g.ly + 2) * g.pxg;
}

// Store psi of node (x, y, z) and its periodic ghost copies.
template <typename R>
__device__ __forceinline__ void store_psi(R* __restrict__ psi, const Geom& g,
                                          int x, int y, int z, R v) {
  const int xs[3] = {x, x == 0 ? g.lx : INT_MIN, x == g.lx - 1 ? -1 : INT_MIN};
  const int ys[3] = {y, y == 0 ? g.ly : INT_MIN, y == g.ly - 1 ? -1 : INT_MIN};
  const int zs[3] = {z, z == 0 ? g.lz : INT_MIN, z == g.lz - 1 ? -1 : INT_MIN};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (zs[c] == INT_MIN) continue;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      if (ys[b] == INT_MIN) continue;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (xs[a] == INT_MIN) continue;
        psi[psi_index(g, xs[a], ys[b], zs[c])] = v;
      }
    }
  }
}

__device__ __forceinline__ long long node_index(const Geom& g, int x, int y,
                                                int z) {
  return ((long long)z * g.ly + y) * g.px + x;
}
__device__ __forceinline__ int wrapc(int v, int n) {
  return v < 0 ? v + n : (v >= n ? v - n : v);
}
__device__ __forceinline__ bool fluid_at(const uint32_t* __restrict__ mask,
                                         const Geom& g, int x, int y, int z) {
  uint32_t w = __ldg(mask + ((long long)z * g.ly + y) * g.wpr + (x >> 5));
  return (w >> (x & 31)) & 1u;
}

// ---- population storage formats --------------------------------------------
// FP32 and FP64 store f_i as is.  FP16 stores h_i = half(f_i - t_i * rho0)
// (shift by the lattice weight times a reference density); arithmetic stays
// in FP32.
template <typename T>
struct Pop;

template <>
struct Pop<float> {
  using Real = float;
  static __device__ __forceinline__ float ld(const float* p, float) {
    return *p;
  }
  static __device__ __forceinline__ void st(float* p, float v, float) {
    *p = v;
  }
};
template <>
struct Pop<double> {
  using Real = double;
  static __device__ __forceinline__ double ld(const double* p, double) {
    return *p;
  }
  static __device__ __forceinline__ void st(double* p, double v, double) {
    *p = v;
  }
};
// The shift is added and subtracted with explicit rounding, so no kernel can
// contract it with the product that forms it (every kernel, scalar or packed,
// stores and reads back the same bits).
template <>
struct Pop<__half> {
  using Real = float;
  static __device__ __forceinline__ float ld(const __half* p, float shift) {
    return __fadd_rn(__half2float(*p), shift);
  }
  static __device__ __forceinline__ void st(__half* p, float v, float shift) {
    *p = __float2half_rn(__fsub_rn(v, shift));
  }
};

// ---- physics parameters ----------------------------------------------------
struct Phys {
  float tau, G, T_Tc, rhol_spinodal, rhog_spinodal, rhos;
  float rho_increment, inject_position;
  int carn_star;
  unsigned long long rho_inject_period;  // 0: never inject
  int inlet_width, outlet_width;
  float rho_inlet, rho_outlet;
  float rho_shift;  // FP16 storage shift (rho0)
  float omega;      // 1/tau rounded once, as the reference's inv_tau
};

// Per-launch step arguments of the reference's multiphaselbm_iteration
// (include/iteration_host.h:56-57).
struct StepArgs {
  long long step;
  int reverse;
  unsigned inject_type;
};

// Rounded arithmetic that the compiler may not contract or reorder, so every
// kernel that inlines collide() produces the same bits.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
// correctly rounded reciprocal: the reference's (float)(1.0 / rho)
__device__ __forceinline__ float rrcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double rrcp(double a) { return __drcp_rn(a); }

__device__ __forceinline__ float expr(float v) { return expf(v); }
__device__ __forceinline__ double expr(double v) { return exp(v); }

// dPress, include/iteration_device.cuh:7-27
template <typename R>
__device__ __forceinline__ R pressure_of(const Phys& p, R rho) {
  if (p.carn_star) {
    const R a = R(1.0), b = R(4.0), Rg = R(1.0), Tc = R(0.0943);
    const R T = rmul(R(p.T_Tc), Tc);
    const R eta = rdiv(rmul(b, rho), R(4.0));
    const R eta2 = rmul(eta, eta), eta3 = rmul(eta2, eta), rho2 = rmul(rho, rho);
    const R ome = rsub(R(1.0), eta);
    const R ome3 = rmul(rmul(ome, ome), ome);
    const R num = rsub(radd(radd(R(1), eta), eta2), eta3);
    return rsub(rdiv(rmul(rmul(rmul(rho, Rg), T), num), ome3), rmul(a, rho2));
  }
  const R cs2 = R(1.0 / 3.0);
  const R psi = rsub(R(1.0), expr(-rho));
  return radd(rmul(cs2, rho), rmul(rdiv(rmul(cs2, R(p.G)), R(2)), rmul(psi, psi)));
}

// dPsi, include/iteration_device.cuh:31-38
template <typename R>
__device__ __forceinline__ R psi_of(const Phys& p, R rho) {
  if (p.carn_star) {
    const R cs2 = R(1.0 / 3.0);
    const R pr = pressure_of<R>(p, rho);
    return sqrt(rdiv(rmul(R(2.0), rsub(pr, rmul(cs2, rho))), rmul(cs2, R(p.G))));
  }
  return rsub(R(1.0), expr(-rho));
}

// 0: interior fluid node, 1: inlet slab, 2: outlet slab (drainage boundary,
// held at fixed density; absent from the reference, defined by this library).
__device__ __forceinline__ int bc_kind(const Phys& p, const Geom& g, int x) {
  return x < p.inlet_width ? 1 : (x >= g.lx - p.outlet_width ? 2 : 0);
}

// Density injection of compute_density, include/iteration_device.cuh:46-59.
template <typename R>
__device__ __forceinline__ R inject(const Phys& p, const Geom& g,
                                    const StepArgs& s, int y, R d) {
  if (p.rho_inject_period != 0 &&
      (float)y < p.inject_position * (float)g.ly &&
      (unsigned long long)s.step % p.rho_inject_period == 0ull) {
    const R inc = rmul(R(p.rho_increment), R(s.reverse));
    switch (s.inject_type) {
      case 0: d = radd(d, inc); break;
      case 1: if (d < R(p.rhol_spinodal)) d = radd(d, inc); break;
      case 2: if (d > R(p.rhol_spinodal)) d = radd(d, inc); break;
      default: break;
    }
  }
  return d;
}

}  // namespace mlbm
