// update_tma.cuh -- the update pass of the two-pass time step: force,
// velocity shift, BGK and AA store for every fluid node, with the psi tiles
// the Shan-Chen force reads staged into shared memory by TMA.
//
// Each block owns a 32 x By tile of the (x, y) plane and a chunk of Dz
// planes, and walks the chunk along z.  psi of planes z-1, z, z+1 (tile plus
// a one-node halo) sits in a ring of four shared-memory slots; while plane z
// is updated, one thread has already issued the bulk tensor copy
// (cp.async.bulk.tensor.3d) of plane z+2 into the fourth slot, completing on
// that slot's mbarrier.  psi is stored with ghost layers (psi_index), so the
// halo box of any tile is one rectangle of the tensor, periodic boundaries
// included; rows past the last tile's end are outside the tensor and come
// back zero-filled (they are not used).  The box starts at x0 - 4 (16-byte
// aligned) and is 40 columns wide.
//
// Shared memory: kRing slots of round_up((By+2) * 40 * sizeof(R), 128) bytes
// plus 128 bytes of alignment slack (update_smem_bytes).
//
// mbarrier waits are bounded: a wait that runs out raises the error flag;
// the block then finishes the plane without storing and returns at the next
// barrier, so no thread is left behind at a barrier, after thread 0 has
// waited (bounded again) for the copies still in flight.
#pragma once

#include <cuda.h>

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

constexpr int kBoxX = 40;  // psi columns x0-4 .. x0+35 of a 32-wide tile
constexpr int kRing = 4;   // psi plane slots

__host__ __device__ constexpr size_t update_smem_bytes(int By, size_t esz) {
  return kRing * ((((size_t)(By + 2) * kBoxX * esz) + 127) / 128 * 128) + 128;
}

struct ZMarch {
  int By;    // tile rows (block = 32 x By threads)
  int Dz;    // planes per block
  int ntx, nty, nzc;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map,
                                            int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

template <typename T, int PHASE, bool WRITE_U>
__global__ void __launch_bounds__(256)
    k_update_zm(T* __restrict__ pop, const uint32_t* __restrict__ nbw,
                float* __restrict__ vel, int* __restrict__ err, Geom g,
                Phys p, StepArgs a, ZMarch zm,
                const __grid_constant__ CUtensorMap psi_map) {
  using R = typename Pop<T>::Real;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[kRing];
  const int wy = zm.By + 2;
  const unsigned slot_bytes = (unsigned)(wy * kBoxX * sizeof(R));
  // bulk tensor copies land on 128-byte aligned shared memory: align the
  // ring base and give every slot a 128-byte multiple stride
  const int slot_elems = (int)(((slot_bytes + 127u) & ~127u) / sizeof(R));
  const uint32_t base_off = smem_addr(smem_raw);
  R* ring = reinterpret_cast<R*>(smem_raw + ((128u - (base_off & 127u)) & 127u));

  int b = blockIdx.x;
  const int tix = b % zm.ntx;
  b /= zm.ntx;
  const int tiy = b % zm.nty;
  const int zc = b / zm.nty;
  const int x0 = tix * 32, y0 = tiy * zm.By;
  const int z0 = zc * zm.Dz, z1 = min(z0 + zm.Dz, g.lz);
  const int tid = threadIdx.x;
  const int x = x0 + (tid & 31), ly_ = tid >> 5, y = y0 + ly_;
  const bool valid = x < g.lx && y < g.ly;
  const R shift = R(p.rho_shift);

  // plane q (q in [z0-1, z1]) lives in slot (q + 1) & 3; its fill has parity
  // ((q - z0 + 1) >> 2) & 1.
  auto slot_of = [](int q) { return (q + 1) & (kRing - 1); };
  auto parity_of = [&](int q) { return (unsigned)(((q - z0 + 1) >> 2) & 1); };
  auto issue = [&](int q) {
    uint64_t* bar = &bars[slot_of(q)];
    mbar_expect_tx(bar, slot_bytes);
    tma_load_3d(ring + slot_of(q) * slot_elems, &psi_map, x0, y0, q + 1, bar);
  };
  if (tid == 0) {
    for (int s = 0; s < kRing; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int issued_hi = z0 + 1;  // the last plane whose copy thread 0 issued
  if (tid == 0) {
    issue(z0 - 1);
    issue(z0);
    issue(z0 + 1);
  }
  auto wait_plane = [&](int q) -> bool {
    long long spins = 0;
    while (!mbar_try_wait(&bars[slot_of(q)], parity_of(q)))
      if (++spins > (1LL << 24)) {
        atomicExch(err, 1);
        return false;
      }
    return true;
  };

  bool ok = wait_plane(z0 - 1) & wait_plane(z0);
  for (int z = z0; z < z1; ++z) {
    if (tid == 0 && z + 2 <= z1) {
      // order the generic-proxy reads of this slot (previous plane, before
      // the last barrier) before the bulk copy overwrites it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(z + 2);
      issued_hi = z + 2;
    }
    const int n = valid ? (int)node_index(g, x, y, z) : 0;
    const uint32_t nb = valid ? nbw[n] : 0u;
    Nbr nbr;
    R f[Q];
    const bool fluid = (nb & NB_SELF) != 0;
    if (fluid) {
      nbr.init(g, x, y, z);
      if (nb_kind(nb))
        slab_populations<R>(R(slab_density(p, nb_kind(nb))), f);
      else
        gather<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
    }
    ok = wait_plane(z + 1) && ok;
    if (fluid && ok) {
      R ux = R(0), uy = R(0), uz = R(0);
      if (!nb_kind(nb)) {
        const R d = sum_density<R>(p, g, a, y, f);
        const R* pm = ring + slot_of(z - 1) * slot_elems;
        const R* p0 = ring + slot_of(z) * slot_elems;
        const R* pp = ring + slot_of(z + 1) * slot_elems;
        const int c = (ly_ + 1) * kBoxX + (tid & 31) + 4;
        collide<R>(
            p, d, p0[c],
            [&](int i) {
              const R* pl = ez(i) < 0 ? pm : (ez(i) > 0 ? pp : p0);
              return pl[c + ey(i) * kBoxX + ex(i)];
            },
            f, ux, uy, uz);
      }
      if (WRITE_U) {
        vel[3 * (long long)n] = (float)ux;
        vel[3 * (long long)n + 1] = (float)uy;
        vel[3 * (long long)n + 2] = (float)uz;
      }
      scatter<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
    }
    // the slot of plane z-1 is refilled next iteration: all reads done first
    if (__syncthreads_or(!ok)) {
      // a wait ran out: leave no bulk copy in flight into this block's
      // shared memory (each ring slot's last issued plane, bounded again)
      if (tid == 0)
        for (int q = max(z0 - 1, issued_hi - (kRing - 1)); q <= issued_hi; ++q)
          wait_plane(q);
      return;
    }
  }
}

}  // namespace mlbm
