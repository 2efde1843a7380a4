// band.cuh -- the one-pass time step over the fluid-only population layout
// (compact.cuh), with two population buffers.
//
// The two-pass step reads every population twice per step: once to form rho
// and psi of all nodes, once more to collide, because the Shan-Chen force of
// a node needs psi of its 18 neighbours at the same time level.  Here each
// launch reads buffer A (pre-collision populations of step t, held in the
// "local" form of AA phase 1: f_i(x, t) at slot i of node x) and writes
// buffer B (the same form for step t + 1, by pushing f*_i(x) to slot i of
// x + e_i, or to slot opp(i) of x itself when x + e_i is solid: halfway
// bounce-back).  A is never written during the launch, so a block may read
// any node's populations at any time, and no block waits for another.
//
// Work item = one band of rows [y0, y1) of every plane of a chunk [z0, z1).
// A block marches the chunk plane by plane (even chunks upward, odd ones
// downward, so a plane shared by two chunks is visited by both at the start
// or both at the end of their marches and comes from DRAM once).  Its warps
// are split in two groups:
//   density warps  form rho and psi of the band's rows plus one halo row on
//                  either side (periodic) for each plane of the march into a
//                  ring of kBandSlots shared-memory psi planes;
//   update warps   update the band's own rows of plane z once psi of planes
//                  z - 1, z, z + 1 is in the ring: force, collision, push.
// The groups hand ring slots over through mbarriers (full: the density warps
// have written the plane; empty: the update warps are done with it), so the
// density warps run up to kBandSlots - 3 planes ahead: their DRAM reads
// overlap the update warps' arithmetic instead of alternating with it.  The
// halo rows belong to the neighbouring bands, whose blocks read them at about
// the same time, and the update re-reads rows the density warps have just
// loaded: both come from L2, so DRAM sees every population about once per
// step.
//
// Every wait is bounded in time: a wait that runs out (wait_ns) raises the
// error flag and its group leaves the kernel; the other group's waits then
// run out too, so the launch always ends.  `stall` (a test of that path)
// makes block 0's update warps wait on a barrier nothing arrives at.
//
// Per node the arithmetic is the two-pass kernels': rho summed in order
// i = 0..18 plus injection, psi_of, collide2 of pair.cuh (two nodes per
// thread in packed FP32), the drainage slabs' rest equilibrium.  Results are
// bit-identical to the two-pass kernels, whose step from phase 1 reads and
// writes the same values at other addresses.
//
// Neighbours that are solid contribute psi(rhos) (wall adhesion,
// include/iteration_device.cuh:69-152): the density warps write psi(rhos)
// at the solid positions of every ring plane, so the update reads all 18
// neighbours from shared memory alike.
#pragma once

#include "compact2.cuh"
#include "update_tma.cuh"

namespace mlbm {

constexpr int kBandD = 128;  // density warps' threads
constexpr int kBandU = 128;  // update warps' threads
constexpr int kBandThreads = kBandD + kBandU;
constexpr int kBandSlots = 6;

// Shared memory of a block: 2 * kBandSlots mbarriers, then kBandSlots planes
// of (hmax + 2) rows of (lx + 2) psi values (ghost columns 0 and lx + 1).
constexpr size_t kBandBarBytes = 2 * kBandSlots * sizeof(uint64_t) + 16;
__host__ __device__ inline size_t band_smem_bytes(int hmax, int lx) {
  return kBandBarBytes + (size_t)kBandSlots * (hmax + 2) * (lx + 2) * sizeof(float);
}

// First compact index of row y of plane z (y in [0, ly]; row ly is the next
// plane's first row, past the odd plane's hole).
__device__ __forceinline__ int band_row_start(const uint2* __restrict__ wtab,
                                              const Geom& g, int z, int y) {
  return (int)__ldg(&wtab[((long long)z * g.ly + y) * g.wpr].y);
}

// One population slot of a pair of nodes from the read-only buffer.
template <typename T>
struct BandLd;
template <>
struct BandLd<float> {
  static __device__ __forceinline__ float2 ld2(const float* p, float) {
    return __ldg(reinterpret_cast<const float2*>(p));
  }
};
template <>
struct BandLd<__half> {
  static __device__ __forceinline__ float2 ld2(const __half* p, float s) {
    return p_add(__half22float2(__ldg(reinterpret_cast<const __half2*>(p))),
                 p_dup(s));
  }
};

template <typename T>
__device__ __forceinline__ void band_gather(const T* __restrict__ A,
                                            uint32_t cs, int k, float shift,
                                            float2 (&f)[Q]) {
#pragma unroll
  for (int i = 0; i < Q; ++i)
    f[i] = BandLd<T>::ld2(A + (uint32_t)i * cs + (uint32_t)k,
                          shift * weight<float>(i));
}

// Decoded node of a pair lane.
struct BandNode {
  uint32_t nb;
  int x, y, kind;
};
__device__ __forceinline__ BandNode band_node(uint2 ci) {
  BandNode n;
  n.nb = ci.x;
  n.x = (int)(ci.y & 2047u);
  n.y = (int)((ci.y >> 11) & 2047u);
  n.kind = nb_kind(ci.x);
  return n;
}

__device__ __forceinline__ void band_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ unsigned long long band_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase of `bar` with parity `parity`; false (error flag set)
// once wait_ns nanoseconds have passed.
__device__ __forceinline__ bool band_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long wait_ns,
                                          int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = band_clock_ns();
  while (!mbar_try_wait(bar, parity))
    if (band_clock_ns() - t0 > wait_ns) {
      atomicExch(err, 1);
      return false;
    }
  return true;
}

struct BandShape {
  int nb, nc;  // bands along y, chunks along z
  int hmax;    // rows of the tallest band
};

template <typename T, bool WRITE_RHO, bool WRITE_U>
__global__ void __launch_bounds__(kBandThreads, 2)
    k_band(const T* __restrict__ A, T* __restrict__ B, uint32_t cs,
           const uint2* __restrict__ cinfo, const uint2* __restrict__ wtab,
           float* __restrict__ rho_out, float* __restrict__ vel,
           int* __restrict__ err, Geom g, Phys p, StepArgs a, bool inj,
           BandShape s, unsigned long long wait_ns, bool stall) {
  extern __shared__ __align__(16) unsigned char band_smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(band_smem);
  uint64_t* empty = full + kBandSlots;
  uint64_t* never = empty + kBandSlots;  // the stall test's barrier
  float* sp = reinterpret_cast<float*>(band_smem + kBandBarBytes);
  const int band = blockIdx.x % s.nb, chunk = blockIdx.x / s.nb;
  const int y0 = (int)((long long)band * g.ly / s.nb);
  const int y1 = (int)((long long)(band + 1) * g.ly / s.nb);
  const int z0 = (int)((long long)chunk * g.lz / s.nc);
  const int z1 = (int)((long long)(chunk + 1) * g.lz / s.nc);
  const int nplanes = z1 - z0;
  // even chunks march up the planes, odd ones down
  const int dir = (chunk & 1) ? -1 : 1;
  const int zfirst = dir > 0 ? z0 : z1 - 1;  // first plane updated
  const int P = g.lx + 2;               // psi row pitch in shared memory
  const int SE = (s.hmax + 2) * P;      // psi plane
  const int rows = y1 - y0;
  const float shift = p.rho_shift;
  // all rows when the band and its halo wrap onto themselves
  const bool all_rows = rows + 2 >= g.ly;

  if (threadIdx.x == 0) {
    for (int k = 0; k < kBandSlots; ++k) {
      mbar_init(&full[k], kBandD);
      mbar_init(&empty[k], kBandU);
    }
    mbar_init(never, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const float psi_solid = psi_of<float>(p, p.rhos);
  if (threadIdx.x < kBandD) {
    // ---- density warps: planes j = 0 .. nplanes + 1 of the march --------
    const int td = threadIdx.x;
    for (int j = 0; j < nplanes + 2; ++j) {
      const int k = j % kBandSlots;
      // the slot's previous plane (j - kBandSlots) released by the update
      if (j >= kBandSlots &&
          !band_wait(&empty[k], (unsigned)((j / kBandSlots - 1) & 1), wait_ns, err))
        return;
      const int zz = zfirst + (j - 1) * dir;
      const int zw = zz < 0 ? zz + g.lz : (zz >= g.lz ? zz - g.lz : zz);
      float* slot = sp + k * SE;
      int ra[2], rb[2], nr = 1;
      if (all_rows) {
        ra[0] = 0; rb[0] = g.ly;
      } else if (y0 == 0) {
        ra[0] = 0; rb[0] = y1 + 1; ra[1] = g.ly - 1; rb[1] = g.ly; nr = 2;
      } else if (y1 == g.ly) {
        ra[0] = y0 - 1; rb[0] = g.ly; ra[1] = 0; rb[1] = 1; nr = 2;
      } else {
        ra[0] = y0 - 1; rb[0] = y1 + 1;
      }
      // psi(rhos) at the solid positions of the slot's rows (wall
      // adhesion: a solid neighbour contributes psi(rhos))
      for (int jr = 0; jr < rows + 2; ++jr) {
        int yy = y0 - 1 + jr;
        yy = yy < 0 ? yy + g.ly : (yy >= g.ly ? yy % g.ly : yy);
        const uint2* wrow = wtab + ((long long)zw * g.ly + yy) * g.wpr;
        float* row = slot + jr * P;
        for (int x = td; x < g.lx; x += kBandD) {
          if ((__ldg(&wrow[x >> 5].x) >> (x & 31)) & 1u) continue;
          row[x + 1] = psi_solid;
          if (x == 0) row[g.lx + 1] = psi_solid;
          if (x == g.lx - 1) row[0] = psi_solid;
        }
      }
      for (int r = 0; r < nr; ++r) {
        const int kf = band_row_start(wtab, g, zw, ra[r]);
        const int ke = band_row_start(wtab, g, zw, rb[r]);
        for (int t = (kf & ~1) + 2 * td; t < ke; t += 2 * kBandD) {
          const BandNode na = band_node(__ldg(cinfo + t));
          const BandNode nbn = band_node(__ldg(cinfo + t + 1));
          const bool va = t >= kf && (na.nb & NB_SELF);
          const bool vb = t + 1 < ke && (nbn.nb & NB_SELF);
          if (!va && !vb) continue;
          float2 f[Q];
          if ((va && !na.kind) || (vb && !nbn.kind)) {
            band_gather<T>(A, cs, t, shift, f);
          } else {
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] = p_dup(0.f);
          }
          float2 d = p_dup(0.f);
#pragma unroll
          for (int i = 0; i < Q; ++i) d = p_add(d, f[i]);
          d.x = na.kind ? slab_density(p, na.kind) : inject_on(p, g, a, inj, na.y, d.x);
          d.y = nbn.kind ? slab_density(p, nbn.kind) : inject_on(p, g, a, inj, nbn.y, d.y);
          // a row's shared-memory rows: j = y - (y0 - 1) (mod ly), and
          // j + ly when the band wraps onto itself
          auto put = [&](const BandNode& n, float v) {
            int jr = n.y - y0 + 1;
            if (jr < 0) jr += g.ly;
            if (jr >= g.ly) jr -= g.ly;
            for (; jr < rows + 2; jr += g.ly) {
              float* row = slot + jr * P;
              row[n.x + 1] = v;
              if (n.x == 0) row[g.lx + 1] = v;
              if (n.x == g.lx - 1) row[0] = v;
            }
          };
          if (va) put(na, psi_of<float>(p, d.x));
          if (vb) put(nbn, psi_of<float>(p, d.y));
        }
      }
      band_arrive(&full[k]);
    }
    return;
  }

  // ---- update warps: plane u of the march needs march planes u, u+1, u+2 --
  const int tu = threadIdx.x - kBandD;
  if (stall && blockIdx.x == 0 && !band_wait(never, 0u, wait_ns, err)) return;
  for (int u = 0; u < nplanes; ++u) {
    for (int j = u == 0 ? 0 : u + 2; j <= u + 2; ++j)
      if (!band_wait(&full[j % kBandSlots], (unsigned)((j / kBandSlots) & 1),
                     wait_ns, err))
        return;
    const int z = zfirst + u * dir;
    const float* s0 = sp + ((u + 1) % kBandSlots) * SE;
    const float* sm = sp + ((dir > 0 ? u : u + 2) % kBandSlots) * SE;   // z - 1
    const float* spl = sp + ((dir > 0 ? u + 2 : u) % kBandSlots) * SE;  // z + 1
    const int kf = band_row_start(wtab, g, z, y0);
    const int ke = band_row_start(wtab, g, z, y1);
    for (int t = (kf & ~1) + 2 * tu; t < ke; t += 2 * kBandU) {
      BandNode na = band_node(__ldg(cinfo + t));
      BandNode nbn = band_node(__ldg(cinfo + t + 1));
      const bool va = t >= kf && (na.nb & NB_SELF);
      const bool vb = t + 1 < ke && (nbn.nb & NB_SELF);
      if (!va && !vb) continue;
      float2 f[Q];
      if ((va && !na.kind) || (vb && !nbn.kind)) {
        band_gather<T>(A, cs, t, shift, f);
      } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = p_dup(0.f);
      }
      // a lane outside the band (or a hole) computes a copy of the other
      // lane and stores nothing
      if (!va) {
        na = nbn;
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i].x = f[i].y;
      }
      if (!vb) {
        nbn = na;
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i].y = f[i].x;
      }
      float2 d = p_dup(0.f);
#pragma unroll
      for (int i = 0; i < Q; ++i) d = p_add(d, f[i]);
      d.x = na.kind ? slab_density(p, na.kind) : inject_on(p, g, a, inj, na.y, d.x);
      d.y = nbn.kind ? slab_density(p, nbn.kind) : inject_on(p, g, a, inj, nbn.y, d.y);
      float2 ux, uy, uz;
      {
        const int ca = (na.y - y0 + 1) * P + na.x + 1;
        const int cb = (nbn.y - y0 + 1) * P + nbn.x + 1;
        collide2(
            p, d, make_float2(s0[ca], s0[cb]),
            [&](int i) {
              const float* pl = ez(i) < 0 ? sm : (ez(i) > 0 ? spl : s0);
              const int o = ey(i) * P + ex(i);
              return make_float2(pl[ca + o], pl[cb + o]);
            },
            f, ux, uy, uz);
      }
      if (na.kind) {
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i].x = rmul(weight<float>(i), d.x);
        ux.x = uy.x = uz.x = 0.f;
      }
      if (nbn.kind) {
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i].y = rmul(weight<float>(i), d.y);
        ux.y = uy.y = uz.y = 0.f;
      }
      // push f*_d to slot d of x + e_d, or to slot opp(d) of x itself
      // (halfway bounce-back) when x + e_d is solid
      auto push = [&](int k, const BandNode& n, int lane) {
        int nk[Q];
        neighbour_ranks(wtab, g, k, n.x, n.y, z, nk);
        if (WRITE_RHO) rho_out[node_index(g, n.x, n.y, z)] = lane ? d.y : d.x;
        if (WRITE_U) {
          const long long m = 3 * node_index(g, n.x, n.y, z);
          vel[m] = lane ? ux.y : ux.x;
          vel[m + 1] = lane ? uy.y : uy.x;
          vel[m + 2] = lane ? uz.y : uz.x;
        }
        PopPair<T>::st1(B + k, lane ? f[0].y : f[0].x, shift * weight<float>(0));
#pragma unroll
        for (int e = 1; e < Q; ++e) {
          const bool fl = (n.nb >> opp(e)) & 1u;
          const uint32_t adr = fl ? (uint32_t)e * cs + (uint32_t)nk[e]
                                  : (uint32_t)opp(e) * cs + (uint32_t)k;
          PopPair<T>::st1(B + adr, lane ? f[e].y : f[e].x,
                          shift * weight<float>(e));
        }
      };
      if (va) push(t, na, 0);
      if (vb) push(t + 1, nbn, 1);
    }
    band_arrive(&empty[u % kBandSlots]);
  }
}

}  // namespace mlbm
