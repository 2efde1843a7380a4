// kernels.cuh -- per-node building blocks of the D3Q19 Shan-Chen update and
// the two-pass time-step kernels.
//
// One lattice buffer, updated in place with the AA access pattern.  The
// stored state alternates between two forms:
//   phase 0 ("own/opposite"): post-collision f*_i(x) sits at pop[opp(i)][x]
//   phase 1 ("pushed"):       post-collision f*_i(x) sits at pop[i][x+e_i]
//                             (at pop[opp(i)][x] when x+e_i is solid)
// A step from phase 0 gathers from the neighbours and pushes to them; a step
// from phase 1 is purely local.  In both, the set of addresses a node reads
// is exactly the set it writes, so the update is race-free in place.  Both
// forms realise the reference's pull streaming with halfway bounce-back
// (include/iteration_device.cuh:252-271, include/iteration_kernel.cuh:65-118):
//   f_i(x, t+1) = f*_i(x - e_i, t)    if x - e_i is fluid
//               = f*_opp(i)(x, t)      otherwise.
//
// Every step is two passes:
//   density pass  (compute_density, include/iteration_device.cuh:40-63):
//                 rho = sum_i f_i (+ injection) for every fluid node, psi(rho);
//   update pass   (compute_force / compute_velocity / post_collision,
//                 include/iteration_device.cuh:69-206): Shan-Chen force from
//                 psi of the 18 neighbours, velocity shift, BGK, store.
// The update pass recomputes the same rho bit for bit from the same loads.
//
// Per-node neighbour word (built once by k_build_nbr): bit 0 = the node is
// fluid; bit i (1..18) = the pull source x - e_i is fluid; bits 19-20 = the
// drainage slab kind (0 interior, 1 inlet, 2 outlet).
#pragma once

#include "lattice.cuh"

namespace mlbm {

constexpr uint32_t NB_SELF = 1u;

// Output flags of one step launch: rho and psi fields, velocity field.
enum { OUT_NONE = 0, OUT_RHO = 1, OUT_VEL = 2 };
__host__ __device__ constexpr int nb_kind(uint32_t nb) { return (nb >> 19) & 3; }

// Neighbour indices of one node: the index of (x+dx, y+dy, z+dz) is
// n + dx + dy*px + dz*ly*px (the displacement part is the same for every
// thread of a launch) plus a per-thread correction for each axis that wraps
// around the periodic boundary; a D3Q19 direction has at most two nonzero
// components, so an index costs one or two integer adds.  Node indices fit
// 32 bits (checked when the lattice is created).
struct Nbr {
  int n, px, pz;            // own index, row pitch, plane pitch
  int cxm, cxp, cym, cyp, czm, czp;  // wrap corrections for -1 / +1 moves
  __device__ __forceinline__ void init(const Geom& g, int x, int y, int z) {
    px = g.px;
    pz = g.ly * g.px;
    n = z * pz + y * px + x;
    cxm = x == 0 ? g.lx : 0;
    cxp = x == g.lx - 1 ? -g.lx : 0;
    cym = y == 0 ? g.ly * px : 0;
    cyp = y == g.ly - 1 ? -g.ly * px : 0;
    czm = z == 0 ? g.lz * pz : 0;
    czp = z == g.lz - 1 ? -g.lz * pz : 0;
  }
  __device__ __forceinline__ int idx(int dx, int dy, int dz) const {
    int v = n + dx + dy * px + dz * pz;
    if (dx) v += dx < 0 ? cxm : cxp;
    if (dy) v += dy < 0 ? cym : cyp;
    if (dz) v += dz < 0 ? czm : czp;
    return v;
  }
};

// Gather the 19 pre-collision populations of a fluid node for a step that
// starts in `PHASE` (see the header comment).
template <typename T, int PHASE>
__device__ __forceinline__ void gather(const T* __restrict__ pop,
                                       long long plane, const Nbr& a,
                                       uint32_t nb, int n,
                                       typename Pop<T>::Real shift,
                                       typename Pop<T>::Real (&f)[Q]) {
  using R = typename Pop<T>::Real;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R s = shift * weight<R>(i);
    int src = n, slot = i;
    if (PHASE == 0 && i != 0 && ((nb >> i) & 1u)) {
      src = a.idx(-ex(i), -ey(i), -ez(i));
      slot = opp(i);
    }
    const T* base = pop + (long long)slot * plane;
    f[i] = Pop<T>::ld(base + src, s);
  }
}

// Store the 19 post-collision populations of a fluid node for a step that
// started in `PHASE`.
template <typename T, int PHASE>
__device__ __forceinline__ void scatter(T* __restrict__ pop, long long plane,
                                        const Nbr& a, uint32_t nb, int n,
                                        typename Pop<T>::Real shift,
                                        const typename Pop<T>::Real (&f)[Q]) {
  using R = typename Pop<T>::Real;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R s = shift * weight<R>(i);
    int dst = n, slot = opp(i);
    // x + e_i is fluid  <=>  the pull source of direction opp(i) is fluid
    if (PHASE == 0 && i != 0 && ((nb >> opp(i)) & 1u)) {
      dst = a.idx(ex(i), ey(i), ez(i));
      slot = i;
    }
    T* base = pop + (long long)slot * plane;
    Pop<T>::st(base + dst, f[i], s);
  }
}

// rho of an interior fluid node from its pre-collision populations, summed in
// the reference's order i = 0..18, plus injection.
template <typename R>
__device__ __forceinline__ R sum_density(const Phys& p, const Geom& g,
                                         const StepArgs& s, int y,
                                         const R (&f)[Q]) {
  R d = R(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
  return inject<R>(p, g, s, y, d);
}

__device__ __forceinline__ float slab_density(const Phys& p, int kind) {
  return kind == 1 ? p.rho_inlet : p.rho_outlet;
}

// Force, velocity shift and BGK relaxation of one interior fluid node
// (include/iteration_device.cuh:69-206).  psi_nb(i) returns psi at x + e_i.
template <typename R, typename PsiNb>
__device__ __forceinline__ void collide(const Phys& p, R d, R psi_self,
                                        PsiNb psi_nb, R (&f)[Q], R& ux, R& uy,
                                        R& uz) {
  // F = -G psi(x) sum_{i=1..18} w_i psi(x + e_i) e_i, terms in order i
  R sx = R(0), sy = R(0), sz = R(0);
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const R wp = rmul(weight<R>(i), psi_nb(i));
    if (ex(i)) sx = ex(i) > 0 ? radd(sx, wp) : rsub(sx, wp);
    if (ey(i)) sy = ey(i) > 0 ? radd(sy, wp) : rsub(sy, wp);
    if (ez(i)) sz = ez(i) > 0 ? radd(sz, wp) : rsub(sz, wp);
  }
  const R gp = rmul(-R(p.G), psi_self);
  const R Fx = rmul(gp, sx), Fy = rmul(gp, sy), Fz = rmul(gp, sz);
  // u = (sum_i f_i e_i + tau F) / rho
  ux = R(0);
  uy = R(0);
  uz = R(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if (ex(i)) ux = ex(i) > 0 ? radd(ux, f[i]) : rsub(ux, f[i]);
    if (ey(i)) uy = ey(i) > 0 ? radd(uy, f[i]) : rsub(uy, f[i]);
    if (ez(i)) uz = ez(i) > 0 ? radd(uz, f[i]) : rsub(uz, f[i]);
  }
  const R tau = R(p.tau);
  const R inv_rho = rrcp(d);
  ux = rmul(rfma(tau, Fx, ux), inv_rho);
  uy = rmul(rfma(tau, Fy, uy), inv_rho);
  uz = rmul(rfma(tau, Fz, uz), inv_rho);
  const R usq15 =
      rmul(R(1.5), rfma(uz, uz, rfma(uy, uy, rmul(ux, ux))));
  const R omega = R(p.omega);
  // BGK, include/iteration_device.cuh:162-174:
  //   f_i += (t_i rho (1 + 3 eu + 4.5 eu^2 - 1.5 u^2) - f_i) / tau
  // evaluated for the pairs (i, opp(i)), whose eu differ only in sign.
  const R base = rsub(R(1), usq15);
  const R wd0 = rmul(weight<R>(0), d), wd1 = rmul(weight<R>(1), d),
          wd2 = rmul(weight<R>(4), d);
  f[0] = rfma(rsub(rmul(wd0, base), f[0]), omega, f[0]);
#pragma unroll
  for (int i = 1; i <= 9; ++i) {
    R eu = R(0);
    if (ex(i)) eu = ex(i) > 0 ? radd(eu, ux) : rsub(eu, ux);
    if (ey(i)) eu = ey(i) > 0 ? radd(eu, uy) : rsub(eu, uy);
    if (ez(i)) eu = ez(i) > 0 ? radd(eu, uz) : rsub(eu, uz);
    const R sym = rfma(rmul(R(4.5), eu), eu, base);
    const R anti = rmul(R(3), eu);
    const R wd = (i <= 3) ? wd1 : wd2;
    const R feq_i = rmul(wd, radd(sym, anti));
    const R feq_o = rmul(wd, rsub(sym, anti));
    f[i] = rfma(rsub(feq_i, f[i]), omega, f[i]);
    f[opp(i)] = rfma(rsub(feq_o, f[opp(i)]), omega, f[opp(i)]);
  }
}

// Rest equilibrium of a drainage-slab node (its post-collision populations).
template <typename R>
__device__ __forceinline__ void slab_populations(R d, R (&f)[Q]) {
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = rmul(weight<R>(i), d);
}

// ---- neighbour words ---------------------------------------------------------
static __global__ void k_build_nbr(const uint32_t* __restrict__ mask,
                            uint32_t* __restrict__ nbw, Geom g, Phys p) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  uint32_t w = 0;
  if (fluid_at(mask, g, x, y, z)) {
    w = NB_SELF;
    for (int i = 1; i < Q; ++i)
      if (fluid_at(mask, g, wrapc(x - ex(i), g.lx), wrapc(y - ey(i), g.ly),
                   wrapc(z - ez(i), g.lz)))
        w |= 1u << i;
    w |= (uint32_t)bc_kind(p, g, x) << 19;
  }
  nbw[node_index(g, x, y, z)] = w;
}

// ---- two-pass kernels -----------------------------------------------------------
// blockDim (32, 4): a warp covers 32 x-consecutive nodes of one row.
template <typename T, int PHASE, bool WRITE_RHO>
__global__ void __launch_bounds__(128)
    k_density(const T* __restrict__ pop, const uint32_t* __restrict__ nbw,
              typename Pop<T>::Real* __restrict__ rho,
              typename Pop<T>::Real* __restrict__ psi, Geom g, Phys p,
              StepArgs s) {
  using R = typename Pop<T>::Real;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  const int n = (int)node_index(g, x, y, z);
  const uint32_t nb = nbw[n];
  if (!(nb & NB_SELF)) return;
  R d;
  if (nb_kind(nb)) {
    d = R(slab_density(p, nb_kind(nb)));
  } else {
    Nbr a;
    a.init(g, x, y, z);
    R f[Q];
    gather<T, PHASE>(pop, g.plane, a, nb, n, R(p.rho_shift), f);
    d = sum_density<R>(p, g, s, y, f);
  }
  if (WRITE_RHO) rho[n] = d;
  store_psi<R>(psi, g, x, y, z, psi_of<R>(p, d));
}

// ---- initialisation (multiphaselbm_init, include/iteration_kernel.cuh:9-29) --
// rho_in holds the initial density of every node in the internal layout.
// f_i = t_i rho at every node; solids get rho = rhos (psi(rhos) follows).
template <typename T>
__global__ void k_init(T* __restrict__ pop, const uint32_t* __restrict__ mask,
                       const float* __restrict__ rho_in,
                       typename Pop<T>::Real* __restrict__ rho,
                       typename Pop<T>::Real* __restrict__ psi, Geom g,
                       Phys p) {
  using R = typename Pop<T>::Real;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  const long long n = node_index(g, x, y, z);
  const R r0 = R(rho_in[n]);
  const R shift = R(p.rho_shift);
#pragma unroll
  for (int i = 0; i < Q; ++i)
    Pop<T>::st(pop + i * g.plane + n, weight<R>(i) * r0, shift * weight<R>(i));
  const R r = fluid_at(mask, g, x, y, z) ? r0 : R(p.rhos);
  rho[n] = r;
  store_psi<R>(psi, g, x, y, z, psi_of<R>(p, r));
}

}  // namespace mlbm
