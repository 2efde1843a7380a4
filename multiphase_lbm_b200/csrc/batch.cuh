// batch.cuh -- many independent lattices advanced by one persistent launch
// per pass: the batched density pass and the batched update pass.
//
// Every domain keeps its own geometry, parameters, AA phase and step origin
// (DomainDesc).  Its work is cut into items -- density: a 32 x By tile of one
// plane; update: a 32 x By tile over Dz consecutive planes -- and the items
// of all domains form one list, domain after domain (prefix offsets).  A
// persistent grid walks the list (item = block + k * grid); the domain of an
// item is found by binary search over the prefix offsets held in shared
// memory.  The per-node arithmetic is the single-lattice kernels' (gather,
// sum_density, collide, scatter), so a domain advanced in a batch is bit
// identical to the same domain advanced alone.
//
// The update pass reads psi of the 18 neighbours straight from the
// ghost-padded psi array (psi_index): the ghost layers make every neighbour
// a constant offset, periodic boundaries included.
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

constexpr int kMaxBatch = 2048;  // domains per batch (prefix array in smem)

struct DomainDesc {
  Geom g;
  Phys p;
  void* pop;
  const uint32_t* nbw;
  void* psi;
  void* rho;
  float* vel;
  int phase_base;            // AA phase at batch step s = (phase_base + s) & 1
  long long step_origin;     // domain step = batch step - step_origin
  int ntx, nty_d, nty_u, nzc;  // tiles: x, y (density rows), y (update rows), z chunks
};

struct BatchArgs {
  int ndomains;
  int By_d, By_u, Dz;
  int reverse;
  unsigned inject_type;
  int write_rho;  // last step of an iterate call: density pass writes rho
};

// Largest d with prefix[d] <= t (prefix[0] = 0, prefix[n] = total).
__device__ __forceinline__ int find_domain(const long long* pre, int n,
                                           long long t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename T, int PHASE>
__device__ __forceinline__ void batch_density_node(const DomainDesc& d,
                                                   const StepArgs& s, int x,
                                                   int y, int z, bool wr) {
  using R = typename Pop<T>::Real;
  const Geom& g = d.g;
  const int n = (int)node_index(g, x, y, z);
  const uint32_t nb = d.nbw[n];
  if (!(nb & NB_SELF)) return;
  R dd;
  if (nb_kind(nb)) {
    dd = R(slab_density(d.p, nb_kind(nb)));
  } else {
    Nbr nbr;
    nbr.init(g, x, y, z);
    R f[Q];
    gather<T, PHASE>(static_cast<const T*>(d.pop), g.plane, nbr, nb, n,
                     R(d.p.rho_shift), f);
    dd = sum_density<R>(d.p, g, s, y, f);
  }
  if (wr) static_cast<R*>(d.rho)[n] = dd;
  store_psi<R>(static_cast<R*>(d.psi), g, x, y, z, psi_of<R>(d.p, dd));
}

template <typename T, int PHASE>
__device__ __forceinline__ void batch_update_node(const DomainDesc& d,
                                                  const StepArgs& s, int x,
                                                  int y, int z) {
  using R = typename Pop<T>::Real;
  const Geom& g = d.g;
  const int n = (int)node_index(g, x, y, z);
  const uint32_t nb = d.nbw[n];
  if (!(nb & NB_SELF)) return;
  T* pop = static_cast<T*>(d.pop);
  const R shift = R(d.p.rho_shift);
  Nbr nbr;
  nbr.init(g, x, y, z);
  R f[Q];
  if (nb_kind(nb)) {
    slab_populations<R>(R(slab_density(d.p, nb_kind(nb))), f);
  } else {
    gather<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
    const R dd = sum_density<R>(d.p, g, s, y, f);
    const R* ps = static_cast<const R*>(d.psi) + psi_index(g, x, y, z);
    const long long sy = g.pxg, sz = (long long)(g.ly + 2) * g.pxg;
    R ux, uy, uz;
    collide<R>(
        d.p, dd, __ldg(ps),
        [&](int i) { return __ldg(ps + ex(i) + ey(i) * sy + ez(i) * sz); }, f,
        ux, uy, uz);
  }
  scatter<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
}

// item -> (domain, tile) with the prefix offsets staged in shared memory
#define MLBM_BATCH_PROLOGUE(PRE)                                      \
  __shared__ long long s_pre[kMaxBatch + 1];                          \
  for (int k = threadIdx.x; k <= a.ndomains; k += blockDim.x)         \
    s_pre[k] = PRE[k];                                                \
  __syncthreads();                                                    \
  const long long total = s_pre[a.ndomains];

template <typename T>
__global__ void __launch_bounds__(256)
    k_batch_density(const DomainDesc* __restrict__ dom,
                    const long long* __restrict__ pre,
                    const long long* __restrict__ step_dev, int step_delta,
                    BatchArgs a) {
  MLBM_BATCH_PROLOGUE(pre)
  const long long bstep = *step_dev + step_delta;
  const int lxi = threadIdx.x & 31, lyi = threadIdx.x >> 5;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const int di = find_domain(s_pre, a.ndomains, t);
    const DomainDesc& d = dom[di];
    long long r = t - s_pre[di];
    const int tx = (int)(r % d.ntx);
    r /= d.ntx;
    const int ty = (int)(r % d.nty_d);
    const int z = (int)(r / d.nty_d);
    const int x = tx * 32 + lxi, y = ty * a.By_d + lyi;
    if (x >= d.g.lx || y >= d.g.ly) continue;
    const StepArgs s{bstep - d.step_origin, a.reverse, a.inject_type};
    if (((d.phase_base + bstep) & 1) == 0)
      batch_density_node<T, 0>(d, s, x, y, z, a.write_rho);
    else
      batch_density_node<T, 1>(d, s, x, y, z, a.write_rho);
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_batch_update(const DomainDesc* __restrict__ dom,
                   const long long* __restrict__ pre,
                   const long long* __restrict__ step_dev, int step_delta,
                   BatchArgs a) {
  MLBM_BATCH_PROLOGUE(pre)
  const long long bstep = *step_dev + step_delta;
  const int lxi = threadIdx.x & 31, lyi = threadIdx.x >> 5;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const int di = find_domain(s_pre, a.ndomains, t);
    const DomainDesc& d = dom[di];
    long long r = t - s_pre[di];
    const int tx = (int)(r % d.ntx);
    r /= d.ntx;
    const int ty = (int)(r % d.nty_u);
    const int zc = (int)(r / d.nty_u);
    const int x = tx * 32 + lxi, y = ty * a.By_u + lyi;
    if (x >= d.g.lx || y >= d.g.ly) continue;
    const StepArgs s{bstep - d.step_origin, a.reverse, a.inject_type};
    const int z0 = zc * a.Dz, z1 = min(z0 + a.Dz, d.g.lz);
    const bool ph0 = ((d.phase_base + bstep) & 1) == 0;
    for (int z = z0; z < z1; ++z) {
      if (ph0) batch_update_node<T, 0>(d, s, x, y, z);
      else batch_update_node<T, 1>(d, s, x, y, z);
    }
  }
}

}  // namespace mlbm
