// pair.cuh -- the per-node work of the compact (fluid-only) kernels done for
// two consecutive fluid nodes per thread with Blackwell's packed FP32
// instructions.
//
// A thread owns the fluid nodes k and k + 1 (k even).  Their populations of
// one slot are adjacent in the compact layout, so in the local AA phase a
// slot of both nodes is one 8-byte load or store (4 bytes in FP16), and all
// arithmetic runs on float2 pairs with the packed fma.rn.f32x2 instruction,
// one instruction for both nodes.  Each lane rounds exactly like the scalar
// __fadd_rn / __fsub_rn / __fmul_rn / __fmaf_rn, and the packed code performs
// the operations of collide() (kernels.cuh) in the same order, so every node
// gets the same bits as in the scalar kernels.
//
// Every plane starts at an even compact index (a plane with an odd fluid
// count is followed by a hole: an unused slot whose node word has no fluid
// bit), so a pair never straddles two planes.  A pair whose second slot is a
// hole holds one node: its second lane is made a copy of the first (same
// node, same loads), so every store of that lane repeats a store of the
// first; only the pair store of the local phase writes the second lane, into
// the hole.
//
// AA addressing (kernels.cuh conventions): in both phases, direction d
// (1..18) of a node uses one address A_d for the load of f_opp(d) and for
// the store of f*_d:
//   phase 1: A_d = opp(d) * cs + k;
//   phase 0: A_d = d * cs + k(x + e_d) if x + e_d is fluid, else
//            opp(d) * cs + k (halfway bounce-back);
// and slot 0 uses k.  Offsets are 32-bit: the compact kernels require
// Q * cs < 2^32.
//
// Included by compact2.cuh, after neighbour_ranks().
#pragma once

#include "compact.cuh"
#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

// ---- packed FP32 -----------------------------------------------------------
// Every packed operation is one fma.rn.f32x2 (__ffma2_rn):
//   a + b = fma(a, 1, b),  a - b = fma(b, -1, a),  a * b = fma(a, b, -0),
// each exact up to its one rounding (the products with +-1 are exact, and
// adding -0 leaves a product unchanged, signed zeros included), so every lane
// rounds like the scalar __fadd_rn / __fsub_rn / __fmul_rn.  The constants
// 1, -1 and -0 are read from constant memory: the assembler turns packed
// operations with literal operands back into a multiply and an add and then
// contracts those into one fma (even with .rn), which would round once where
// the scalar code rounds twice.
static __constant__ float2 c_pk_one = {1.f, 1.f};
static __constant__ float2 c_pk_neg_one = {-1.f, -1.f};
static __constant__ float2 c_pk_neg_zero = {-0.f, -0.f};

__device__ __forceinline__ float2 p_dup(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) {
  return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 p_add(float2 a, float2 b) {
  return p_fma(a, c_pk_one, b);
}
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) {
  return p_fma(b, c_pk_neg_one, a);
}
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) {
  return p_fma(a, b, c_pk_neg_zero);
}

// Loads and stores of one population of both nodes of a pair.
template <typename T>
struct PopPair;
template <>
struct PopPair<float> {
  // adjacent pair (k even): one 8-byte access
  static __device__ __forceinline__ float2 ld2(const float* p, float) {
    return *reinterpret_cast<const float2*>(p);
  }
  static __device__ __forceinline__ void st2(float* p, float2 v, float) {
    *reinterpret_cast<float2*>(p) = v;
  }
  static __device__ __forceinline__ float ld1(const float* p, float) { return *p; }
  static __device__ __forceinline__ void st1(float* p, float v, float) { *p = v; }
};
template <>
struct PopPair<__half> {
  static __device__ __forceinline__ float2 ld2(const __half* p, float s) {
    return p_add(__half22float2(*reinterpret_cast<const __half2*>(p)), p_dup(s));
  }
  static __device__ __forceinline__ void st2(__half* p, float2 v, float s) {
    *reinterpret_cast<__half2*>(p) = __float22half2_rn(p_sub(v, p_dup(s)));
  }
  static __device__ __forceinline__ float ld1(const __half* p, float s) {
    return __fadd_rn(__half2float(*p), s);
  }
  static __device__ __forceinline__ void st1(__half* p, float v, float s) {
    *p = __float2half_rn(__fsub_rn(v, s));
  }
};

// ---- one pair of fluid nodes -----------------------------------------------
struct PairNode {
  int k;        // compact index
  int x, y, z;
  uint32_t nb;  // neighbour word
  int kind;     // drainage slab kind
};

__device__ __forceinline__ PairNode pair_node(const uint2* __restrict__ cinfo,
                                              int k) {
  const uint2 ci = __ldg(cinfo + k);
  PairNode n;
  n.k = k;
  n.nb = ci.x;
  n.x = (int)(ci.y & 2047u);
  n.y = (int)((ci.y >> 11) & 2047u);
  n.z = (int)(ci.y >> 22);
  n.kind = nb_kind(ci.x);
  return n;
}

// A_d of one node in AA phase 0 (see the header comment); A[0] = k.
__device__ __forceinline__ void aa_addresses0(const uint2* __restrict__ wtab,
                                              const Geom& g, uint32_t cs,
                                              const PairNode& n,
                                              uint32_t (&A)[Q]) {
  int nk[Q];
  neighbour_ranks(wtab, g, n.k, n.x, n.y, n.z, nk);
  A[0] = (uint32_t)n.k;
#pragma unroll
  for (int d = 1; d < Q; ++d) {
    const bool fl = (n.nb >> opp(d)) & 1u;  // x + e_d is fluid
    A[d] = fl ? (uint32_t)d * cs + (uint32_t)nk[d]
              : (uint32_t)opp(d) * cs + (uint32_t)n.k;
  }
}

// Pre-collision populations of the pair: f[i] = (node a, node b).
template <typename T, int PHASE>
__device__ __forceinline__ void pair_gather(const T* cpop, uint32_t cs, int k,
                                            const uint32_t (&A)[Q],
                                            const uint32_t (&B)[Q], float shift,
                                            float2 (&f)[Q]) {
  if (PHASE == 1) {
    f[0] = PopPair<T>::ld2(cpop + k, shift * weight<float>(0));
#pragma unroll
    for (int d = 1; d < Q; ++d)
      f[opp(d)] = PopPair<T>::ld2(cpop + (uint32_t)opp(d) * cs + (uint32_t)k,
                                  shift * weight<float>(d));
  } else {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const float s = shift * weight<float>(d);
      const int i = opp(d);
      f[i].x = PopPair<T>::ld1(cpop + A[d], s);
      f[i].y = PopPair<T>::ld1(cpop + B[d], s);
    }
  }
}

template <typename T, int PHASE>
__device__ __forceinline__ void pair_scatter(T* cpop, uint32_t cs, int k,
                                             const uint32_t (&A)[Q],
                                             const uint32_t (&B)[Q],
                                             float shift, const float2 (&f)[Q]) {
  if (PHASE == 1) {
    PopPair<T>::st2(cpop + k, f[0], shift * weight<float>(0));
#pragma unroll
    for (int d = 1; d < Q; ++d)
      PopPair<T>::st2(cpop + (uint32_t)opp(d) * cs + (uint32_t)k, f[d],
                      shift * weight<float>(d));
  } else {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const float s = shift * weight<float>(d);
      PopPair<T>::st1(cpop + A[d], f[d].x, s);
      PopPair<T>::st1(cpop + B[d], f[d].y, s);
    }
  }
}

// Force, velocity shift and BGK of two interior fluid nodes: collide() of
// kernels.cuh, operation for operation, in packed form.  psi_nb(i) returns
// psi at x + e_i of both nodes.
template <typename PsiNb>
__device__ __forceinline__ void collide2(const Phys& p, float2 d, float2 psi_self,
                                         PsiNb psi_nb, float2 (&f)[Q],
                                         float2& ux, float2& uy, float2& uz) {
  float2 sx = p_dup(0.f), sy = p_dup(0.f), sz = p_dup(0.f);
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const float2 wp = p_mul(p_dup(weight<float>(i)), psi_nb(i));
    if (ex(i)) sx = ex(i) > 0 ? p_add(sx, wp) : p_sub(sx, wp);
    if (ey(i)) sy = ey(i) > 0 ? p_add(sy, wp) : p_sub(sy, wp);
    if (ez(i)) sz = ez(i) > 0 ? p_add(sz, wp) : p_sub(sz, wp);
  }
  const float2 gp = p_mul(p_dup(-p.G), psi_self);
  const float2 Fx = p_mul(gp, sx), Fy = p_mul(gp, sy), Fz = p_mul(gp, sz);
  ux = p_dup(0.f);
  uy = p_dup(0.f);
  uz = p_dup(0.f);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if (ex(i)) ux = ex(i) > 0 ? p_add(ux, f[i]) : p_sub(ux, f[i]);
    if (ey(i)) uy = ey(i) > 0 ? p_add(uy, f[i]) : p_sub(uy, f[i]);
    if (ez(i)) uz = ez(i) > 0 ? p_add(uz, f[i]) : p_sub(uz, f[i]);
  }
  const float2 tau = p_dup(p.tau);
  const float2 inv_rho = make_float2(rrcp(d.x), rrcp(d.y));
  ux = p_mul(p_fma(tau, Fx, ux), inv_rho);
  uy = p_mul(p_fma(tau, Fy, uy), inv_rho);
  uz = p_mul(p_fma(tau, Fz, uz), inv_rho);
  const float2 usq15 =
      p_mul(p_dup(1.5f), p_fma(uz, uz, p_fma(uy, uy, p_mul(ux, ux))));
  const float2 omega = p_dup(p.omega);
  const float2 base = p_sub(p_dup(1.f), usq15);
  const float2 wd0 = p_mul(p_dup(weight<float>(0)), d),
               wd1 = p_mul(p_dup(weight<float>(1)), d),
               wd2 = p_mul(p_dup(weight<float>(4)), d);
  f[0] = p_fma(p_sub(p_mul(wd0, base), f[0]), omega, f[0]);
#pragma unroll
  for (int i = 1; i <= 9; ++i) {
    float2 eu = p_dup(0.f);
    if (ex(i)) eu = ex(i) > 0 ? p_add(eu, ux) : p_sub(eu, ux);
    if (ey(i)) eu = ey(i) > 0 ? p_add(eu, uy) : p_sub(eu, uy);
    if (ez(i)) eu = ez(i) > 0 ? p_add(eu, uz) : p_sub(eu, uz);
    const float2 sym = p_fma(p_mul(p_dup(4.5f), eu), eu, base);
    const float2 anti = p_mul(p_dup(3.f), eu);
    const float2 wd = (i <= 3) ? wd1 : wd2;
    const float2 feq_i = p_mul(wd, p_add(sym, anti));
    const float2 feq_o = p_mul(wd, p_sub(sym, anti));
    f[i] = p_fma(p_sub(feq_i, f[i]), omega, f[i]);
    f[opp(i)] = p_fma(p_sub(feq_o, f[opp(i)]), omega, f[opp(i)]);
  }
}

// psi reader of the update pass, given psi_index() positions: the float psi
// array through the read-only path (psi complete before the launch).
// ready() is called once before the first psi read.
struct PsiPlain {
  const float* psi;
  __device__ __forceinline__ void ready() const {}
  __device__ __forceinline__ float self(uint32_t i) const { return __ldg(psi + i); }
  __device__ __forceinline__ float nb(uint32_t i, int) const { return __ldg(psi + i); }
};

// Programmatic dependent launch.  A step kernel launched with the
// programmatic-serialization attribute may start while the kernel before it
// in the stream is still running; pdl_gate() waits until that kernel has
// completed and its memory is visible (griddepcontrol.wait), then lets the
// next kernel of the stream start the same way (launch_dependents).  Work
// before the gate may only read what the kernel before does not write (the
// node table, the AA addresses; in the update pass also the populations,
// which the density pass only reads).  Without the attribute both
// instructions return at once.
template <bool PDL>
__device__ __forceinline__ void pdl_gate() {
  if (PDL) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  }
}

// The two nodes of pair k (k even) and whether the second one exists.
struct Pair {
  PairNode a, b;
  bool two;
};

__device__ __forceinline__ Pair load_pair(const uint2* __restrict__ cinfo, int k,
                                          int nfluid) {
  Pair q;
  q.a = pair_node(cinfo, k);
  q.b = pair_node(cinfo, k + 1);  // k + 1 < nfluid: the slot count is even
  q.two = (q.b.nb & NB_SELF) != 0u;
  if (!q.two) q.b = q.a;
  return q;
}

// Pre-collision populations of pair q (both phases), with the second lane a
// copy of the first for a single-node pair.
template <typename T, int PHASE, bool GATE = false>
__device__ __forceinline__ void pair_load(const T* cpop, uint32_t cs,
                                          const uint2* __restrict__ wtab,
                                          const Geom& g, const Pair& q,
                                          float shift, uint32_t (&A)[Q],
                                          uint32_t (&B)[Q], float2 (&f)[Q]) {
  if (PHASE == 0) {
    aa_addresses0(wtab, g, cs, q.a, A);
    aa_addresses0(wtab, g, cs, q.b, B);
  }
  pdl_gate<GATE>();
  if (q.a.kind && q.b.kind) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = p_dup(0.f);
  } else {
    pair_gather<T, PHASE>(cpop, cs, q.a.k, A, B, shift, f);
  }
  if (!q.two) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i].y = f[i].x;
  }
}

// rho of both nodes: sum in the order i = 0..18 (+ injection), or the slab
// density.
__device__ __forceinline__ float2 pair_rho(const Phys& p, const Geom& g,
                                           const StepArgs& a, bool inj,
                                           const Pair& q, const float2 (&f)[Q]) {
  float2 d = p_dup(0.f);
#pragma unroll
  for (int i = 0; i < Q; ++i) d = p_add(d, f[i]);
  d.x = q.a.kind ? slab_density(p, q.a.kind) : inject_on(p, g, a, inj, q.a.y, d.x);
  d.y = q.b.kind ? slab_density(p, q.b.kind) : inject_on(p, g, a, inj, q.b.y, d.y);
  return d;
}

// Density pass of one pair (the work of k_cdensity for two nodes).
template <typename T, int PHASE, bool WRITE_RHO, bool PDL = false>
__device__ __forceinline__ void pair_density(const T* cpop, uint32_t cs,
                                             const uint2* __restrict__ cinfo,
                                             const uint2* __restrict__ wtab,
                                             int k, int nfluid, float* rho_out,
                                             float* psi, const Geom& g,
                                             const Phys& p, const StepArgs& a,
                                             bool inj) {
  const Pair q = load_pair(cinfo, k, nfluid);
  uint32_t A[Q], B[Q];
  float2 f[Q];
  pair_load<T, PHASE, PDL>(cpop, cs, wtab, g, q, p.rho_shift, A, B, f);
  const float2 d = pair_rho(p, g, a, inj, q, f);
  if (WRITE_RHO) {
    rho_out[node_index(g, q.a.x, q.a.y, q.a.z)] = d.x;
    rho_out[node_index(g, q.b.x, q.b.y, q.b.z)] = d.y;
  }
  store_psi<float>(psi, g, q.a.x, q.a.y, q.a.z, psi_of<float>(p, d.x));
  if (q.two) store_psi<float>(psi, g, q.b.x, q.b.y, q.b.z, psi_of<float>(p, d.y));
}

// Update pass of one pair (the work of k_cupdate for two nodes).
template <typename T, int PHASE, bool WRITE_U, class PsiR, bool PDL = false>
__device__ __forceinline__ void pair_update(T* cpop, uint32_t cs,
                                            const uint2* __restrict__ cinfo,
                                            const uint2* __restrict__ wtab,
                                            int k, int nfluid, const PsiR& pr,
                                            float* vel, const Geom& g,
                                            const Phys& p, const StepArgs& a,
                                            bool inj) {
  const Pair q = load_pair(cinfo, k, nfluid);
  uint32_t A[Q], B[Q];
  float2 f[Q];
  // The gather/push step (phase 0) parks its 2 x 19 addresses in shared
  // memory between the gather and the push: held in registers across the
  // collision they leave too few for 3 CTAs per SM.  Each node's addresses
  // are parked right after its own gather, so only 19 are live at a time.
  // (k_cupdate: 1-D blocks of kC2Threads.)
  __shared__ uint32_t parked[PHASE == 0 ? 2 * Q : 1][PHASE == 0 ? kC2Threads : 1];
  if (PHASE == 0) {
    aa_addresses0(wtab, g, cs, q.a, A);
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      f[opp(e)].x = PopPair<T>::ld1(cpop + A[e], p.rho_shift * weight<float>(e));
      parked[e][threadIdx.x] = A[e];
    }
    aa_addresses0(wtab, g, cs, q.b, A);  // q.b is q.a for a one-node pair
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      f[opp(e)].y = PopPair<T>::ld1(cpop + A[e], p.rho_shift * weight<float>(e));
      parked[Q + e][threadIdx.x] = A[e];
    }
  } else {
    pair_load<T, PHASE>(cpop, cs, wtab, g, q, p.rho_shift, A, B, f);
  }
  pdl_gate<PDL>();  // psi and the population stores come from / go after it
  const float2 d = pair_rho(p, g, a, inj, q, f);
  float2 ux, uy, uz;
  {
    const uint32_t pa = (uint32_t)psi_index(g, q.a.x, q.a.y, q.a.z);
    const uint32_t pb = (uint32_t)psi_index(g, q.b.x, q.b.y, q.b.z);
    const int sy = g.pxg, sz = (g.ly + 2) * g.pxg;
    pr.ready();
    collide2(
        p, d, make_float2(pr.self(pa), pr.self(pb)),
        [&](int i) {
          const int o = ex(i) + ey(i) * sy + ez(i) * sz;
          return make_float2(pr.nb(pa + o, i), pr.nb(pb + o, i));
        },
        f, ux, uy, uz);
  }
  if (q.a.kind) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i].x = rmul(weight<float>(i), d.x);
    ux.x = uy.x = uz.x = 0.f;
  }
  if (q.b.kind) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i].y = rmul(weight<float>(i), d.y);
    ux.y = uy.y = uz.y = 0.f;
  }
  if (WRITE_U) {
    const long long na = node_index(g, q.a.x, q.a.y, q.a.z);
    const long long nb = node_index(g, q.b.x, q.b.y, q.b.z);
    vel[3 * na] = ux.x;
    vel[3 * na + 1] = uy.x;
    vel[3 * na + 2] = uz.x;
    vel[3 * nb] = ux.y;
    vel[3 * nb + 1] = uy.y;
    vel[3 * nb + 2] = uz.y;
  }
  if (PHASE == 0) {
    const volatile uint32_t(*pk)[PHASE == 0 ? kC2Threads : 1] = parked;
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      A[e] = pk[e][threadIdx.x];
      B[e] = pk[Q + e][threadIdx.x];
    }
  }
  pair_scatter<T, PHASE>(cpop, cs, k, A, B, p.rho_shift, f);
}



// ---- one node per thread (AA phase 0) -----------------------------------------
// The density pass of the gather step: one node per thread (on pairs it
// measured slower at 64 and at 80 registers).  Holes (no fluid bit) are
// skipped.
template <typename T, bool WRITE_RHO, bool PDL = false>
__device__ __forceinline__ void node_density0(const T* cpop, uint32_t cs,
                                              const uint2* __restrict__ cinfo,
                                              const uint2* __restrict__ wtab,
                                              int k, float* rho_out, float* psi,
                                              const Geom& g, const Phys& p,
                                              const StepArgs& a, bool inj) {
  const PairNode n = pair_node(cinfo, k);
  if (!(n.nb & NB_SELF)) return;
  float d;
  if (n.kind) {
    pdl_gate<PDL>();
    d = slab_density(p, n.kind);
  } else {
    uint32_t A[Q];
    aa_addresses0(wtab, g, cs, n, A);
    pdl_gate<PDL>();
    float f[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e)
      f[opp(e)] = PopPair<T>::ld1(cpop + A[e], p.rho_shift * weight<float>(e));
    d = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
    d = inject_on(p, g, a, inj, n.y, d);
  }
  if (WRITE_RHO) rho_out[node_index(g, n.x, n.y, n.z)] = d;
  store_psi<float>(psi, g, n.x, n.y, n.z, psi_of<float>(p, d));
}

}  // namespace mlbm
