// batch_compact.cuh -- the batched time step over the compact (fluid-only)
// layout: the density pass and the update pass of every domain of a batch,
// one launch each, with the per-node work of the single-lattice compact
// kernels (pair.cuh), so a domain advanced in a batch is bit-identical to the
// same domain advanced alone.
//
// Each domain owns a contiguous range of blocks.  The AA phase of a domain
// at batch step s is phase_base ^ (s & 1).  The density pass runs one node
// per thread in the gather step and one pair per thread in the local step,
// so a domain's block count depends on the parity of s: two block-prefix
// tables, one per parity, and the launch grid covers the larger total.  The
// update pass runs one pair per thread in both phases (one table).  The
// batch step s is read from the device counter (graph replays advance it),
// so a captured graph stays valid for every start parity.
#pragma once

#include "batch.cuh"
#include "compact2.cuh"
#include "lattice.cuh"

namespace mlbm {

constexpr int kBCThreads = 256;

struct CDomain {
  Geom g;
  Phys p;
  void* cpop;                 // [Q][cs] populations (T)
  const uint2* cinfo;         // [cs]
  const uint2* wtab;          // mask word table
  float* psi;
  float* rho;
  uint32_t cs;
  int nfluid;                 // compact slots (even)
  int phase_base;
  long long step_origin;
};

// Domain, local block and AA phase of this block at batch step s; false if
// the block has no work at this parity.
__device__ __forceinline__ bool bc_locate(const long long* __restrict__ pre,
                                          int n, long long s, int& d,
                                          long long& local) {
  const int par = (int)(s & 1);
  const long long* pp = pre + (size_t)par * (n + 1);
  const long long b = blockIdx.x;
  if (b >= pp[n]) return false;
  d = find_domain(pp, n, b);
  local = b - pp[d];
  return true;
}

__device__ __forceinline__ bool bc_inject(const Phys& p, long long dstep) {
  return p.rho_inject_period != 0ull &&
         (unsigned long long)dstep % p.rho_inject_period == 0ull;
}

template <typename T, bool WRITE_RHO>
__global__ void __launch_bounds__(kBCThreads, 3)
    k_batch_cdensity(const CDomain* __restrict__ doms,
                     const long long* __restrict__ pre, int n,
                     const long long* __restrict__ step, int delta, int reverse,
                     unsigned inject_type) {
  const long long s = *step + delta;
  int d;
  long long local;
  if (!bc_locate(pre, n, s, d, local)) return;
  const CDomain& D = doms[d];
  const int ph = D.phase_base ^ (int)(s & 1);
  StepArgs a{s - D.step_origin, reverse, inject_type};
  const bool inj = bc_inject(D.p, a.step);
  const long long t = local * kBCThreads + threadIdx.x;
  if (ph == 0) {
    if (t >= D.nfluid) return;
    node_density0<T, WRITE_RHO>(static_cast<const T*>(D.cpop), D.cs, D.cinfo,
                                D.wtab, (int)t, D.rho, D.psi, D.g, D.p, a, inj);
  } else {
    if (2 * t >= D.nfluid) return;
    pair_density<T, 1, WRITE_RHO>(static_cast<const T*>(D.cpop), D.cs, D.cinfo,
                                  D.wtab, (int)(2 * t), D.nfluid, D.rho, D.psi,
                                  D.g, D.p, a, inj);
  }
}

// upre: the update pass's block prefixes (n + 1 entries, both parities).
// Blocks of kBCThreads = kC2Threads threads, as pair_update's phase-0 form
// requires.
template <typename T>
__global__ void __launch_bounds__(kBCThreads, 3)
    k_batch_cupdate(const CDomain* __restrict__ doms,
                    const long long* __restrict__ upre, int n,
                    const long long* __restrict__ step, int delta, int reverse,
                    unsigned inject_type) {
  static_assert(kBCThreads == kC2Threads, "pair_update's parked addresses");
  const long long s = *step + delta;
  const long long b = blockIdx.x;
  if (b >= upre[n]) return;
  const int d = find_domain(upre, n, b);
  const CDomain& D = doms[d];
  const int ph = D.phase_base ^ (int)(s & 1);
  StepArgs a{s - D.step_origin, reverse, inject_type};
  const bool inj = bc_inject(D.p, a.step);
  const long long k = 2 * ((b - upre[d]) * kBCThreads + threadIdx.x);
  if (k >= D.nfluid) return;
  if (ph == 0)
    pair_update<T, 0, false>(static_cast<T*>(D.cpop), D.cs, D.cinfo, D.wtab,
                             (int)k, D.nfluid, PsiPlain{D.psi}, nullptr, D.g,
                             D.p, a, inj);
  else
    pair_update<T, 1, false>(static_cast<T*>(D.cpop), D.cs, D.cinfo, D.wtab,
                             (int)k, D.nfluid, PsiPlain{D.psi}, nullptr, D.g,
                             D.p, a, inj);
}

}  // namespace mlbm
