// kernels.cuh -- the time-step kernels of the D3Q19 Shan-Chen update.
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
//                 rho = sum_i f_i (+ injection) for every fluid node;
//   update pass   (compute_force / compute_velocity / post_collision,
//                 include/iteration_device.cuh:69-206): Shan-Chen force from
//                 psi(rho) of the 18 neighbours, velocity shift, BGK, store.
// The update pass recomputes the same rho bit for bit from the same loads.
#pragma once

#include "lattice.cuh"

namespace mlbm {

// Load the 19 pre-collision populations of node (x,y,z) for a step that
// starts in `PHASE`.
template <typename T, int PHASE>
__device__ __forceinline__ void load_pre(
    const T* __restrict__ pop, const uint32_t* __restrict__ mask,
    const Geom& g, int x, int y, int z, long long n,
    typename Pop<T>::Real shift, typename Pop<T>::Real (&f)[Q]) {
  using R = typename Pop<T>::Real;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R s = shift * weight<R>(i);
    if (PHASE == 1 || i == 0) {
      f[i] = Pop<T>::ld(pop + i * g.plane + n, s);
    } else {
      const int xs = wrapc(x - ex(i), g.lx), ys = wrapc(y - ey(i), g.ly),
                zs = wrapc(z - ez(i), g.lz);
      if (fluid_at(mask, g, xs, ys, zs))
        f[i] = Pop<T>::ld(pop + opp(i) * g.plane + node_index(g, xs, ys, zs), s);
      else
        f[i] = Pop<T>::ld(pop + i * g.plane + n, s);
    }
  }
}

// Store the 19 post-collision populations of node (x,y,z) for a step that
// started in `PHASE`.
template <typename T, int PHASE>
__device__ __forceinline__ void store_post(
    T* __restrict__ pop, const uint32_t* __restrict__ mask, const Geom& g,
    int x, int y, int z, long long n, typename Pop<T>::Real shift,
    const typename Pop<T>::Real (&f)[Q]) {
  using R = typename Pop<T>::Real;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R s = shift * weight<R>(i);
    if (PHASE == 1 || i == 0) {
      Pop<T>::st(pop + opp(i) * g.plane + n, f[i], s);
    } else {
      const int xd = wrapc(x + ex(i), g.lx), yd = wrapc(y + ey(i), g.ly),
                zd = wrapc(z + ez(i), g.lz);
      if (fluid_at(mask, g, xd, yd, zd))
        Pop<T>::st(pop + i * g.plane + node_index(g, xd, yd, zd), f[i], s);
      else
        Pop<T>::st(pop + opp(i) * g.plane + n, f[i], s);
    }
  }
}

// rho of a fluid node from its pre-collision populations, summed in the
// reference's order i = 0..18, plus injection; fixed at the drainage slabs.
template <typename R>
__device__ __forceinline__ R node_density(const Phys& p, const Geom& g,
                                          const StepArgs& s, int x, int y,
                                          const R (&f)[Q]) {
  const int bc = bc_kind(p, g, x);
  if (bc) return R(bc == 1 ? p.rho_inlet : p.rho_outlet);
  R d = R(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) d += f[i];
  return inject<R>(p, g, s, y, d);
}

// ---- density pass ------------------------------------------------------------
template <typename T, int PHASE>
__global__ void __launch_bounds__(128)
    k_density(const T* __restrict__ pop, const uint32_t* __restrict__ mask,
              typename Pop<T>::Real* __restrict__ rho,
              typename Pop<T>::Real* __restrict__ psi, Geom g, Phys p,
              StepArgs s) {
  using R = typename Pop<T>::Real;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(mask, g, x, y, z)) return;
  const long long n = node_index(g, x, y, z);
  R d;
  if (bc_kind(p, g, x)) {
    R dummy[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) dummy[i] = R(0);
    d = node_density<R>(p, g, s, x, y, dummy);
  } else {
    R f[Q];
    load_pre<T, PHASE>(pop, mask, g, x, y, z, n, R(p.rho_shift), f);
    d = node_density<R>(p, g, s, x, y, f);
  }
  rho[n] = d;
  psi[n] = psi_of<R>(p, d);
}

// ---- update pass -------------------------------------------------------------
template <typename T, int PHASE, bool WRITE_U>
__global__ void __launch_bounds__(128)
    k_update(T* __restrict__ pop, const uint32_t* __restrict__ mask,
             const typename Pop<T>::Real* __restrict__ rho,
             const typename Pop<T>::Real* __restrict__ psi,
             float* __restrict__ vel, Geom g, Phys p, StepArgs s) {
  using R = typename Pop<T>::Real;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(mask, g, x, y, z)) return;
  const long long n = node_index(g, x, y, z);
  const R shift = R(p.rho_shift);
  R f[Q];
  const int bc = bc_kind(p, g, x);
  if (bc) {
    // Drainage slabs: post-collision populations are the rest equilibrium.
    const R d = R(bc == 1 ? p.rho_inlet : p.rho_outlet);
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = weight<R>(i) * d;
    if (WRITE_U) {
      vel[3 * n] = 0.f;
      vel[3 * n + 1] = 0.f;
      vel[3 * n + 2] = 0.f;
    }
    store_post<T, PHASE>(pop, mask, g, x, y, z, n, shift, f);
    return;
  }
  load_pre<T, PHASE>(pop, mask, g, x, y, z, n, shift, f);
  const R d = rho[n];

  // Shan-Chen force, include/iteration_device.cuh:69-152:
  //   F = -G psi(x) sum_{i=1..18} w_i psi(x + e_i) e_i
  R sx = R(0), sy = R(0), sz = R(0);
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const int xn = wrapc(x + ex(i), g.lx), yn = wrapc(y + ey(i), g.ly),
              zn = wrapc(z + ez(i), g.lz);
    const R wp = weight<R>(i) * __ldg(psi + node_index(g, xn, yn, zn));
    if (ex(i)) sx += ex(i) > 0 ? wp : -wp;
    if (ey(i)) sy += ey(i) > 0 ? wp : -wp;
    if (ez(i)) sz += ez(i) > 0 ? wp : -wp;
  }
  const R gp = -R(p.G) * psi[n];
  const R Fx = gp * sx, Fy = gp * sy, Fz = gp * sz;

  // Velocity shift, include/iteration_device.cuh:181-206:
  //   u = (sum_i f_i e_i + tau F) / rho
  R ux = R(0), uy = R(0), uz = R(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if (ex(i)) ux += ex(i) > 0 ? f[i] : -f[i];
    if (ey(i)) uy += ey(i) > 0 ? f[i] : -f[i];
    if (ez(i)) uz += ez(i) > 0 ? f[i] : -f[i];
  }
  const R tau = R(p.tau);
  const R inv_rho = R(1) / d;
  ux = (ux + tau * Fx) * inv_rho;
  uy = (uy + tau * Fy) * inv_rho;
  uz = (uz + tau * Fz) * inv_rho;
  if (WRITE_U) {
    vel[3 * n] = (float)ux;
    vel[3 * n + 1] = (float)uy;
    vel[3 * n + 2] = (float)uz;
  }
  const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
  const R omega = R(1) / tau;

  // BGK relaxation, include/iteration_device.cuh:162-174
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    R eu = R(0);
    if (ex(i)) eu += ex(i) > 0 ? ux : -ux;
    if (ey(i)) eu += ey(i) > 0 ? uy : -uy;
    if (ez(i)) eu += ez(i) > 0 ? uz : -uz;
    const R feq = weight<R>(i) * d *
                  (R(1) + R(3) * eu + R(4.5) * eu * eu - usq15);
    f[i] = f[i] + (feq - f[i]) * omega;
  }
  store_post<T, PHASE>(pop, mask, g, x, y, z, n, shift, f);
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
  psi[n] = psi_of<R>(p, r);
}

}  // namespace mlbm
