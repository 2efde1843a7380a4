// persistent.cuh -- the fused time step: one persistent, cooperative launch
// per lattice step.
//
// Why: the Shan-Chen force at step n needs psi(rho_n) of all 18 neighbours,
// and rho_n is only known once the neighbours' populations have streamed in,
// so every step has two passes over the lattice (density pass P, update pass
// U).  Run as two kernels, U re-reads all populations from DRAM (236 B per
// fluid node instead of 152).  Here both passes run inside one launch, plane
// by plane: the density pass of plane z+L is issued before the update pass
// of plane z, so by the time a block updates plane z its populations were
// read by the density pass a few planes earlier and are still in L2.  DRAM
// then sees one read and one write of each population plus the 4-byte psi.
//
// Schedule.  A work item ("ticket") is a block of By rows x W nodes of one
// z-plane, either its density pass (P) or its update pass (U).  Tickets are
// numbered in slot order: slot s issues P of the s-th plane of the list
// [lz-1, 0, 1, ..., lz-2] and then U of plane s-L.  Block b of the grid
// takes tickets b, b+G, b+2G, ...  U of plane z waits until P of planes
// z-1, z, z+1 (periodic) are complete; P never waits.  Every wait is on a
// ticket with a smaller number, and all G blocks are co-resident
// (cooperative launch), so the earliest unfinished ticket can always run:
// no deadlock.  Waits are bounded (clock-based budget); on expiry a block
// raises the error flag, and every block that sees the flag returns.
//
// Memory ordering.  P blocks store psi with plain stores, then
// __syncthreads(), then one thread issues __threadfence() and increments the
// plane's counter.  The waiting thread polls the counter with an acquire
// load, and after __syncthreads() the block reads psi with L2-only loads
// (__ldcg), which cannot hit a stale L1 line.
//
// Race freedom of the in-place AA update: the set of population addresses a
// node reads is exactly the set it writes, and the sets of different nodes
// are disjoint, so P of one plane and U of another never touch the same
// address; U of a plane runs after P of the same plane (it waits for it).
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

struct Sched {
  int By;          // rows per block item
  int W;           // nodes per row segment (multiple of 32)
  int nseg;        // row segments per row
  int rb_y;        // row blocks per plane along y = ceil(ly / By)
  int R;           // items per plane = rb_y * nseg
  int L;           // slot lag between P of a plane and U of the same plane
  long long total; // tickets per step
  unsigned target; // counter value meaning "plane complete" this launch
  long long budget_cycles;  // wait budget (clock64 cycles)
};

// Output flags of one launch.
enum { OUT_NONE = 0, OUT_RHO = 1, OUT_VEL = 2 };

struct Ticket {
  int is_u;
  int z;
  int rb;
};

__device__ __forceinline__ Ticket decode_ticket(long long t, const Sched& s,
                                                int lz) {
  Ticket k;
  const long long R = s.R, L = s.L;
  long long slot, r;
  int u;
  if (t < L * R) {
    slot = t / R;
    r = t % R;
    u = 0;
  } else {
    const long long t1 = t - L * R;
    const long long mid = (long long)(lz - L) * 2 * R;
    if (t1 < mid) {
      slot = L + t1 / (2 * R);
      const long long q = t1 % (2 * R);
      u = q >= R;
      r = q % R;
    } else {
      const long long t2 = t1 - mid;
      slot = lz + t2 / R;
      r = t2 % R;
      u = 1;
    }
  }
  k.is_u = u;
  k.rb = (int)r;
  if (u) {
    k.z = (int)(slot - L);
  } else {
    // P plane list [lz-1, 0, 1, ..., lz-2]
    k.z = slot == 0 ? lz - 1 : (int)slot - 1;
  }
  return k;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Wait (one thread) until the three planes around z are complete.  Returns
// false when the budget ran out or another block raised the error flag.
__device__ __forceinline__ bool wait_planes(const unsigned* pdone, int* err,
                                            int z, int lz, const Sched& s) {
  const int zm = z == 0 ? lz - 1 : z - 1, zp = z == lz - 1 ? 0 : z + 1;
  const long long t0 = clock64();
  unsigned backoff = 32;
  while (true) {
    if (ld_acquire(pdone + zm) >= s.target && ld_acquire(pdone + z) >= s.target &&
        ld_acquire(pdone + zp) >= s.target)
      return true;
    if (*(volatile int*)err) return false;
    if (clock64() - t0 > s.budget_cycles) {
      atomicExch(err, 1);
      return false;
    }
    __nanosleep(backoff);
    if (backoff < 512) backoff <<= 1;
  }
}

template <typename T, int PHASE, int OUT>
__global__ void __launch_bounds__(512)
    k_step_fused(T* __restrict__ pop, const uint32_t* __restrict__ nbw,
                 typename Pop<T>::Real* __restrict__ psi,
                 typename Pop<T>::Real* __restrict__ rho_out,
                 float* __restrict__ vel, unsigned* __restrict__ pdone,
                 int* __restrict__ err, Geom g, Phys p, StepArgs a, Sched s) {
  using R = typename Pop<T>::Real;
  extern __shared__ unsigned char smem_raw[];
  R* sp = reinterpret_cast<R*>(smem_raw);  // [3][By+2][lx] psi tile
  const int tid = threadIdx.x;
  const int ty = tid / s.W, tx = tid % s.W;
  const int rows = s.By + 2;
  const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  const R shift = R(p.rho_shift);
  __shared__ int s_ok;

  for (long long t = blockIdx.x; t < s.total; t += gridDim.x) {
    const Ticket k = decode_ticket(t, s, g.lz);
    const int y0 = (k.rb / s.nseg) * s.By;
    const int x = (k.rb % s.nseg) * s.W + tx;
    const int y = y0 + ty;
    const int z = k.z;
    const bool valid = x < g.lx && y < g.ly;
    const int n = valid ? (int)node_index(g, x, y, z) : 0;
    const uint32_t nb = valid ? nbw[n] : 0u;
    const bool fluid = (nb & NB_SELF) != 0;
    const int kind = nb_kind(nb);
    if (!k.is_u) {
      // ---- density pass: psi (and rho on output steps) of plane z -----------
      if (fluid) {
        R d;
        if (kind) {
          d = R(slab_density(p, kind));
        } else {
          Nbr nbr;
          nbr.init(g, x, y, z);
          R f[Q];
          gather<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
          d = sum_density<R>(p, g, a, y, f);
        }
        psi[n] = psi_of<R>(p, d);
        if (OUT & OUT_RHO) rho_out[n] = d;
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        atomicAdd(pdone + z, 1u);
      }
    } else {
      // ---- update pass of plane z ---------------------------------------------
      // The populations do not depend on the other blocks' density passes:
      // load them first so their latency overlaps the wait and the psi tile.
      Nbr nbr;
      R f[Q];
      if (fluid) {
        nbr.init(g, x, y, z);
        if (kind)
          slab_populations<R>(R(slab_density(p, kind)), f);
        else
          gather<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
      }
      if (tid == 0) s_ok = wait_planes(pdone, err, z, g.lz, s) ? 1 : 0;
      __syncthreads();
      if (!s_ok) return;
      // psi of planes z-1..z+1, rows y0-1..y0+By, whole rows (x wraps)
      for (int rr = warp; rr < 3 * rows; rr += nwarps) {
        const int zz = wrapc(z - 1 + rr / rows, g.lz);
        const int yy = wrapc(y0 - 1 + rr % rows, g.ly);
        const R* src = psi + node_index(g, 0, yy, zz);
        R* dst = sp + rr * g.lx;
        for (int xx = lane; xx < g.lx; xx += 32) dst[xx] = __ldcg(src + xx);
      }
      __syncthreads();
      if (fluid) {
        R ux = R(0), uy = R(0), uz = R(0);
        if (!kind) {
          const R d = sum_density<R>(p, g, a, y, f);
          const int ry = ty + 1;  // row of (x, y) inside the tile
          collide<R>(
              p, d, sp[(rows + ry) * g.lx + x],
              [&](int i) {
                const int xn = ex(i) < 0 ? nbr.xm : (ex(i) > 0 ? nbr.xp : x);
                return sp[((1 + ez(i)) * rows + ry + ey(i)) * g.lx + xn];
              },
              f, ux, uy, uz);
        }
        if (OUT & OUT_VEL) {
          vel[3 * (long long)n] = (float)ux;
          vel[3 * (long long)n + 1] = (float)uy;
          vel[3 * (long long)n + 2] = (float)uz;
        }
        scatter<T, PHASE>(pop, g.plane, nbr, nb, n, shift, f);
      }
      __syncthreads();  // the psi tile is reused by the next item
    }
  }
}

}  // namespace mlbm
