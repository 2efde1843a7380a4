// wave.cuh -- the time step over the compact (fluid-only) population layout
// as ONE persistent launch that reads the populations from DRAM once.
//
// The two-pass step (compact2.cuh) streams the populations twice per step:
// the density pass needs rho of every node before the update pass may use
// psi(rho) of the 18 neighbours.  Here both passes run inside one launch as
// a wavefront along z.  The fluid nodes of each plane (a contiguous compact
// range, since compact order is z-major) are cut into tiles; the work list
// holds every density tile D(z, j) and update tile U(z, j) in an order where
// the density tiles run `lookahead` planes ahead of the update tiles:
//
//   D(lz-1), D(0) .. D(L), U(0), D(L+1), U(1), D(L+2), ... , U(lz-1)
//
// (D(lz-1) first because U(0) needs psi of the periodic neighbour plane).
// CTAs take work items in list order from a ticket counter; a density tile
// publishes its plane's progress with a release increment of done[z], and an
// update tile of plane z first waits (thread 0, acquire loads, bounded) until
// planes z-1, z, z+1 are complete.  An update tile re-reads populations that
// the density tile of its plane read a few planes earlier, so the second read
// hits L2 and DRAM sees each population once per step.
//
// Correctness of the in-place (AA) update: every node reads and writes only
// its own address set, disjoint from every other node's; U(z) starts after
// D(z) has read the set of every node of plane z, so no density read sees a
// value of the new step.  psi is written (D) and read (U) within the launch,
// so U reads it with ordinary coherent loads, never through the read-only
// (non-coherent) path; the acquire by thread 0 followed by the CTA barrier
// orders those loads after the density tiles' stores.
//
// Deadlock freedom: a CTA holds at most two tickets (the item it works on and
// the next, prefetched), an update tile only waits for density tiles with
// smaller tickets, and density tiles never wait, so every wait ends once the
// CTAs holding earlier tickets (all resident, since they took a ticket) have
// finished them.  The wait is still bounded: past `spin_limit` polls (or at
// once, when the error flag is already set) the CTA sets the error flag and
// skips the tile, and the host reports the step as failed.
//
// Counters: two sets (ticket + done[lz]), used by alternate launches; each
// launch clears the set the next launch uses (its previous user has
// finished: launches on one stream run in order).
//
// Per node pair the work is that of the compact two-pass kernels (pair.cuh),
// with psi read through coherent loads; results are bit-identical to the
// two-pass kernels.  Tiles hold whole pairs: planes start at even compact
// indices and tile sizes are even.
#pragma once

#include "compact.cuh"
#include "compact2.cuh"
#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

constexpr int kWaveThreads = 256;
// CTAs per SM the register allocation is sized for: the gather/scatter step
// (AA phase 0, neighbour ranks) needs more registers than the local step.
template <int PHASE>
constexpr int wave_min_blocks() { return PHASE == 0 ? 2 : 3; }
constexpr int kWaveDensity = 0, kWaveUpdate = 1;

// One work item: plane z, kind (density / update), compact range [k0, k1).
struct WaveItem {
  int z, kind, k0, k1;
};

struct WaveArgs {
  const int4* items;       // [nitems] (z, kind, k0, k1)
  const unsigned* need;    // [lz] density tiles of each plane
  unsigned* ticket;        // [2]
  unsigned* done;          // [2][lz]
  int* err;                // set to 3 when a wait runs out
  int nitems, lz, par;     // par: the counter set of this launch
  unsigned spin_limit;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T, int PHASE, int OUT>
__global__ void __launch_bounds__(kWaveThreads, wave_min_blocks<PHASE>())
    k_cwave(T* cpop, uint32_t cs, int nfluid, const uint2* __restrict__ cinfo,
            const uint2* __restrict__ wtab, float* rho_out, float* psi,
            float* vel, Geom g, Phys p, StepArgs a, bool inj, WaveArgs w) {
  __shared__ int s_item[2];
  const int tid = threadIdx.x;
  // clear the counter set of the next launch
  if (blockIdx.x == 0) {
    unsigned* nd = w.done + (size_t)(w.par ^ 1) * w.lz;
    for (int i = tid; i < w.lz; i += kWaveThreads) nd[i] = 0u;
    if (tid == 0) w.ticket[w.par ^ 1] = 0u;
  }
  unsigned* done = w.done + (size_t)w.par * w.lz;
  unsigned* ticket = w.ticket + w.par;
  int next = 0;
  if (tid == 0) next = (int)atomicAdd(ticket, 1u);
  for (int it = 0;; ++it) {
    if (tid == 0) {
      int t = next;
      if (t < w.nitems) {
        next = (int)atomicAdd(ticket, 1u);  // prefetch the following item
        const int4 item = __ldg(w.items + t);
        if (item.y == kWaveUpdate) {
          const int z = item.x;
          const int zm = z == 0 ? w.lz - 1 : z - 1;
          const int zp = z == w.lz - 1 ? 0 : z + 1;
          const unsigned nm = __ldg(w.need + zm), n0 = __ldg(w.need + z),
                         np = __ldg(w.need + zp);
          unsigned polls = 0;
          while (ld_acquire(done + zm) < nm || ld_acquire(done + z) < n0 ||
                 ld_acquire(done + zp) < np) {
            // give up past the poll limit, or at once when another wait of
            // this lattice has already given up
            if (++polls > w.spin_limit || *(volatile int*)w.err != 0) {
              atomicExch(w.err, 3);
              t = -1;  // skip the tile; the host reports the failed step
              break;
            }
            __nanosleep(64);
          }
        }
      }
      s_item[it & 1] = t;
    }
    __syncthreads();
    const int t = s_item[it & 1];
    if (t >= w.nitems) break;
    if (t < 0) continue;
    const int4 item = __ldg(w.items + t);
    constexpr int per = PHASE == 0 ? 1 : 2;  // nodes per thread
    if (item.y == kWaveDensity) {
#pragma unroll 1
      for (int k = item.z + per * tid; k < item.w; k += per * kWaveThreads) {
        if (PHASE == 0)
          node_density0<T, (OUT & OUT_RHO) != 0>(cpop, cs, cinfo, wtab, k,
                                                 rho_out, psi, g, p, a, inj);
        else
          pair_density<T, 1, (OUT & OUT_RHO) != 0>(cpop, cs, cinfo, wtab, k,
                                                   nfluid, rho_out, psi, g, p,
                                                   a, inj);
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        atomicAdd(done + item.x, 1u);
      }
    } else {
#pragma unroll 1
      for (int k = item.z + per * tid; k < item.w; k += per * kWaveThreads) {
        if (PHASE == 0)
          node_update0<T, (OUT & OUT_VEL) != 0>(cpop, cs, cinfo, wtab, k,
                                                PsiCoherent{psi}, vel, g, p, a,
                                                inj);
        else
          pair_update<T, 1, (OUT & OUT_VEL) != 0>(
              cpop, cs, cinfo, wtab, k, nfluid, PsiCoherent{psi}, vel, g, p, a,
              inj);
      }
    }
  }
}

}  // namespace mlbm
