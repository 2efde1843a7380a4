// persistent.cuh -- the fused time step: one persistent, cooperative launch
// per lattice step that marches through the lattice along z.
//
// Why: the Shan-Chen force at step n needs psi(rho_n) of all 18 neighbours,
// and rho_n is only known once the neighbours' populations have streamed in,
// so every step has two passes over the lattice (density pass P, update pass
// U).  As two kernels, U re-reads every population from DRAM.  Here each
// block owns one Tx x Ty tile of the (x, y) plane for all z and walks the
// planes: iteration `it` runs P of the it-th plane of the list
// [lz-1, 0, 1, ..., lz-2] and U of plane it-L.  U of a plane re-reads
// populations that P of the same plane read L iterations earlier, which are
// still in L2, so DRAM sees one read and one write of each population plus
// the psi values.
//
// Dependencies.  U of plane z needs psi of planes z-1, z, z+1 in the tile and
// a one-node halo, i.e. P of those planes in this tile and in the 8
// neighbouring tiles.  After its P stage a block publishes how many P planes
// it has finished (a per-tile counter, release store); before its U stage it
// waits (acquire loads) until its neighbours have finished the P planes it
// needs.  Those were issued at most L-2 iterations ago (L >= 2 is enough for
// progress; a larger L gives slack), and a P stage never waits, so with all
// tiles' blocks co-resident (cooperative launch, grid = number of tiles)
// every wait ends: by induction on `it`, every block's P stage of iteration
// `it` completes, hence every U stage of iteration `it` completes.  Waits are
// still bounded by a clock budget; on expiry a block raises the error flag
// and every block that sees the flag returns.
//
// psi window.  Shared memory holds psi of three planes for the tile plus its
// halo ring; each U stage loads only the newest plane (from L2, with
// L2-only loads, so no stale L1 line can be read) and reuses the other two.
//
// Race freedom of the in-place AA update: the set of population addresses a
// node reads is exactly the set it writes, and the sets of different nodes
// are disjoint, so stages of different planes or tiles never touch the same
// address; U of a plane runs after P of the same plane (same block, earlier
// iteration).  psi of a plane is written once per launch, before any block
// reads it.
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

struct March {
  int Tx, Ty;        // tile size (Tx a multiple of 32)
  int ntx, nty;      // tiles along x (over the padded row) and y
  int L;             // iteration lag between P and U of the same plane
  unsigned base;     // counter value at the start of this launch
  long long budget_cycles;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Position of plane z in the P list [lz-1, 0, 1, ..., lz-2].
__device__ __forceinline__ int p_pos(int z, int lz) { return z == lz - 1 ? 0 : z + 1; }

template <typename T, int PHASE, int OUT>
__global__ void __launch_bounds__(512)
    k_step_fused(T* __restrict__ pop, const uint32_t* __restrict__ nbw,
                 typename Pop<T>::Real* __restrict__ psi,
                 typename Pop<T>::Real* __restrict__ rho_out,
                 float* __restrict__ vel, unsigned* __restrict__ prog,
                 int* __restrict__ err, Geom g, Phys p, StepArgs a, March s) {
  using R = typename Pop<T>::Real;
  extern __shared__ unsigned char smem_raw[];
  const int wx = s.Tx + 2, wy = s.Ty + 2, wplane = wx * wy;
  R* win = reinterpret_cast<R*>(smem_raw);  // [3][Ty+2][Tx+2] psi window

  const int tile = blockIdx.x;
  const int tix = tile % s.ntx, tiy = tile / s.ntx;
  const int x0 = tix * s.Tx, y0 = tiy * s.Ty;
  const int tid = threadIdx.x;
  const int lxi = tid % s.Tx, lyi = tid / s.Tx;
  const int x = x0 + lxi, y = y0 + lyi;
  const bool valid = x < g.lx && y < g.ly;
  const R shift = R(p.rho_shift);
  const int plane_nodes = g.ly * g.px;

  // neighbouring tiles (periodic tile grid) whose P progress U waits for
  int nbr_tile = tile;
  if (tid < 9) {
    const int dx = tid % 3 - 1, dy = tid / 3 - 1;
    const int ntx = (tix + dx + s.ntx) % s.ntx, nty = (tiy + dy + s.nty) % s.nty;
    nbr_tile = nty * s.ntx + ntx;
  }

  int loaded = 0;  // planes of the psi window loaded so far in this launch
  const int iters = g.lz + s.L;
  for (int it = 0; it < iters; ++it) {
    const int zp = it < g.lz ? (it == 0 ? g.lz - 1 : it - 1) : -1;
    const int zu = it - s.L;
    const bool do_u = zu >= 0 && zu < g.lz;

    // ---- issue the loads of both stages first -----------------------------
    Nbr nbP, nbU;
    uint32_t wP = 0, wU = 0;
    int nP = 0, nU = 0;
    R fP[Q], fU[Q];
    if (zp >= 0 && valid) {
      nP = zp * plane_nodes + y * g.px + x;
      wP = nbw[nP];
      if ((wP & NB_SELF) && !nb_kind(wP)) {
        nbP.init(g, x, y, zp);
        gather<T, PHASE>(pop, g.plane, nbP, wP, nP, shift, fP);
      }
    }
    if (do_u && valid) {
      nU = zu * plane_nodes + y * g.px + x;
      wU = nbw[nU];
      if (wU & NB_SELF) {
        nbU.init(g, x, y, zu);
        if (nb_kind(wU))
          slab_populations<R>(R(slab_density(p, nb_kind(wU))), fU);
        else
          gather<T, PHASE>(pop, g.plane, nbU, wU, nU, shift, fU);
      }
    }

    // ---- P stage: psi (and rho on output steps) of plane zp -----------------
    if (zp >= 0) {
      if (wP & NB_SELF) {
        const R d = nb_kind(wP) ? R(slab_density(p, nb_kind(wP)))
                                : sum_density<R>(p, g, a, y, fP);
        store_psi<R>(psi, g, x, y, zp, psi_of<R>(p, d));
        if (OUT & OUT_RHO) rho_out[nP] = d;
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        st_release(prog + tile, s.base + (unsigned)(it + 1));
      }
    }
    if (!do_u) continue;

    // ---- U stage of plane zu --------------------------------------------------
    // wait for P of planes zu-1, zu, zu+1 in the 9 tiles around this one
    int need = p_pos(zu, g.lz);
    need = max(need, p_pos(zu == 0 ? g.lz - 1 : zu - 1, g.lz));
    need = max(need, p_pos(zu == g.lz - 1 ? 0 : zu + 1, g.lz));
    const unsigned target = s.base + (unsigned)(need + 1);
    bool ok = true;
    if (tid < 9) {
      const long long t0 = clock64();
      unsigned backoff = 32;
      while (ld_acquire(prog + nbr_tile) < target) {
        if (*(volatile int*)err) { ok = false; break; }
        if (clock64() - t0 > s.budget_cycles) {
          atomicExch(err, 1);
          ok = false;
          break;
        }
        __nanosleep(backoff);
        if (backoff < 256) backoff <<= 1;
      }
    }
    // uniform decision for the whole block (barrier + OR)
    if (__syncthreads_or(!ok)) return;
    // refresh the psi window: planes zu-1, zu, zu+1 (only the newest plane
    // after the first U stage)
    for (int k = (loaded == 0 ? -1 : 1); k <= 1; ++k) {
      const int zz = wrapc(zu + k, g.lz);
      const int slot = (zu + k + 3) % 3;
      R* dst = win + slot * wplane;
      for (int j = tid; j < wplane; j += blockDim.x) {
        const int jy = j / wx, jx = j - jy * wx;
        const int gy = wrapc(y0 - 1 + jy, g.ly);
        int gx = x0 - 1 + jx;
        gx = gx < 0 ? gx + g.lx : (gx >= g.lx ? gx - g.lx : gx);
        dst[j] = (gx >= 0 && gx < g.lx) ? __ldcg(psi + psi_index(g, gx, gy, zz))
                                        : R(0);
      }
    }
    loaded = 1;
    __syncthreads();
    if (wU & NB_SELF) {
      R ux = R(0), uy = R(0), uz = R(0);
      if (!nb_kind(wU)) {
        const R d = sum_density<R>(p, g, a, y, fU);
        const int cx = lxi + 1, cy = lyi + 1;
        const int sm = ((zu + 2) % 3) * wplane, s0 = (zu % 3) * wplane,
                  sp1 = ((zu + 1) % 3) * wplane;
        collide<R>(
            p, d, win[s0 + cy * wx + cx],
            [&](int i) {
              const int base = ez(i) < 0 ? sm : (ez(i) > 0 ? sp1 : s0);
              return win[base + (cy + ey(i)) * wx + cx + ex(i)];
            },
            fU, ux, uy, uz);
      }
      if (OUT & OUT_VEL) {
        vel[3 * (long long)nU] = (float)ux;
        vel[3 * (long long)nU + 1] = (float)uy;
        vel[3 * (long long)nU + 2] = (float)uz;
      }
      scatter<T, PHASE>(pop, g.plane, nbU, wU, nU, shift, fU);
    }
  }
}

}  // namespace mlbm
