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
// or both at the end of their marches and comes from DRAM once).  The rows
// y0 - 1 .. y1 of a plane (the band and one halo row on either side,
// periodic) are one or two contiguous ranges of compact indices, so for
// every plane of the march a producer thread copies those ranges of the 19
// population arrays and of the node table into a ring of kBandStages
// shared-memory stages with bulk asynchronous copies (cp.async.bulk,
// completing on the stage's mbarrier), kBandStages planes ahead.  Then
//   density warps  form rho and psi of the staged rows into a ring of
//                  kBandSlots shared-memory psi planes;
//   update warps   take the band's own rows of plane z from the same stage
//                  once psi of planes z - 1, z, z + 1 is in the ring: force,
//                  collision, push to buffer B.
// The bytes in flight are the producer's copies, not loads held in
// registers, so a few warps keep DRAM busy.  The halo rows belong to the
// neighbouring bands, whose blocks copy them at about the same time: L2
// serves the second copy, and DRAM sees every population about once per
// step.  Stages and psi planes are handed over through mbarriers (stage
// full: the copies have landed; stage free: density and update warps are
// done with it; psi full / psi free likewise).
//
// Every wait is bounded in time: a wait that runs out (wait_ns) raises the
// error flag and its group leaves the kernel (the producer first waits, with
// the same bound, for the copies it has in flight); the other groups' waits
// then run out too, so the launch always ends.  `stall` (a test of that
// path) makes block 0's update warps wait on a barrier nothing completes.
//
// Per node the arithmetic is the two-pass kernels': rho summed in order
// i = 0..18 plus injection, psi_of, collide2 of pair.cuh (two nodes per
// thread in packed FP32), the drainage slabs' rest equilibrium.  Results are
// bit-identical to the two-pass kernels, whose step from phase 1 reads and
// writes the same values at other addresses.  Neighbours that are solid
// contribute psi(rhos) (wall adhesion, include/iteration_device.cuh:69-152);
// the node's neighbour word selects it.
#pragma once

#include "compact2.cuh"
#include "update_tma.cuh"

namespace mlbm {

constexpr int kBandP = 32;   // producer warp (one thread issues the copies)
constexpr int kBandD = 128;  // density warps' threads
constexpr int kBandU = 128;  // update warps' threads
constexpr int kBandThreads = kBandP + kBandD + kBandU;
constexpr int kBandSlots = 4;   // psi planes
constexpr int kBandStages = 3;  // staged planes of populations

// Rows y0 - 1 .. y1 of a band (periodic in y) as at most two ranges of rows
// [ra, rb); all rows when the band and its halo wrap onto themselves.
__host__ __device__ inline int band_row_ranges(int ly, int y0, int y1,
                                               int (&ra)[2], int (&rb)[2]) {
  if (y1 - y0 + 2 >= ly) { ra[0] = 0; rb[0] = ly; return 1; }
  if (y0 == 0) { ra[0] = 0; rb[0] = y1 + 1; ra[1] = ly - 1; rb[1] = ly; return 2; }
  if (y1 == ly) { ra[0] = y0 - 1; rb[0] = ly; ra[1] = 0; rb[1] = 1; return 2; }
  ra[0] = y0 - 1; rb[0] = y1 + 1;
  return 1;
}

// Element alignment of staged ranges: bulk copies move multiples of 16
// bytes between 16-byte aligned addresses.
template <typename T>
__host__ __device__ constexpr int band_align() { return 16 / (int)sizeof(T); }

// Bytes of one stage holding `slot` compact slots: 19 population runs and
// the node-table run (uint2), each a multiple of 128 bytes.
template <typename T>
__host__ __device__ inline size_t band_stage_bytes(int slot) {
  return ((size_t)Q * slot * sizeof(T) + 127) / 128 * 128 +
         ((size_t)slot * sizeof(uint2) + 127) / 128 * 128;
}
constexpr size_t kBandBarBytes = 128;  // mbarriers (2 * stages + 2 * slots + 1)
// Shared memory of a block: mbarriers, the psi ring, the stages.
template <typename T>
__host__ __device__ inline size_t band_smem_bytes(int hmax, int lx, int slot) {
  const size_t ring = ((size_t)kBandSlots * (hmax + 2) * (lx + 2) * sizeof(float) +
                       127) / 128 * 128;
  return kBandBarBytes + ring + kBandStages * band_stage_bytes<T>(slot);
}

// First compact index of row y of plane z (y in [0, ly]; row ly is the next
// plane's first row, past the odd plane's hole).
__device__ __forceinline__ int band_row_start(const uint2* __restrict__ wtab,
                                              const Geom& g, int z, int y) {
  return (int)__ldg(&wtab[((long long)z * g.ly + y) * g.wpr].y);
}

// One population slot of a pair of nodes from a stage (shared memory).
template <typename T>
struct StageLd;
template <>
struct StageLd<float> {
  static __device__ __forceinline__ float2 ld2(const float* p, float) {
    return *reinterpret_cast<const float2*>(p);
  }
};
template <>
struct StageLd<__half> {
  static __device__ __forceinline__ float2 ld2(const __half* p, float s) {
    return p_add(__half22float2(*reinterpret_cast<const __half2*>(p)), p_dup(s));
  }
};

// The 19 populations of the pair at stage index `idx` (even).
template <typename T>
__device__ __forceinline__ void stage_gather(const T* st, int slot, int idx,
                                             float shift, float2 (&f)[Q]) {
#pragma unroll
  for (int i = 0; i < Q; ++i)
    f[i] = StageLd<T>::ld2(st + i * slot + idx, shift * weight<float>(i));
}

// One bulk copy global -> shared memory completing on `bar` (16-byte
// aligned addresses, a multiple of 16 bytes).
__device__ __forceinline__ void bulk_copy(void* dst, const void* src,
                                          unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
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
  int slot;    // compact slots a stage holds (multiple of band_align)
};

// The staged ranges of plane zw for the band [y0, y1): compact bounds
// [kf, ke) of each row range, and its aligned start a and stage offset off.
struct BandRanges {
  int n;
  int kf[2], ke[2], a[2], off[2], len[2];
};
template <typename T>
__device__ __forceinline__ BandRanges band_ranges(const uint2* __restrict__ wtab,
                                                  const Geom& g, int zw, int y0,
                                                  int y1) {
  BandRanges r;
  int ra[2], rb[2];
  r.n = band_row_ranges(g.ly, y0, y1, ra, rb);
  int off = 0;
  for (int q = 0; q < r.n; ++q) {
    r.kf[q] = band_row_start(wtab, g, zw, ra[q]);
    r.ke[q] = band_row_start(wtab, g, zw, rb[q]);
    r.a[q] = r.kf[q] & ~(band_align<T>() - 1);
    const int e = (r.ke[q] + band_align<T>() - 1) & ~(band_align<T>() - 1);
    r.len[q] = e - r.a[q];
    r.off[q] = off;
    off += r.len[q];
  }
  return r;
}

template <typename T, bool WRITE_RHO, bool WRITE_U>
__global__ void __launch_bounds__(kBandThreads, 1)
    k_band(const T* __restrict__ A, T* __restrict__ B, uint32_t cs,
           const uint2* __restrict__ cinfo, const uint2* __restrict__ wtab,
           float* __restrict__ rho_out, float* __restrict__ vel,
           int* __restrict__ err, Geom g, Phys p, StepArgs a, bool inj,
           BandShape s, unsigned long long wait_ns, bool stall) {
  extern __shared__ __align__(128) unsigned char band_smem[];
  uint64_t* stage_full = reinterpret_cast<uint64_t*>(band_smem);
  uint64_t* stage_free = stage_full + kBandStages;
  uint64_t* psi_full = stage_free + kBandStages;
  uint64_t* psi_free = psi_full + kBandSlots;
  uint64_t* never = psi_free + kBandSlots;  // the stall test's barrier
  const int P = g.lx + 2;               // psi row pitch in shared memory
  const int SE = (s.hmax + 2) * P;      // psi plane
  float* sp = reinterpret_cast<float*>(band_smem + kBandBarBytes);
  unsigned char* stages = band_smem + kBandBarBytes +
                          ((size_t)kBandSlots * SE * sizeof(float) + 127) / 128 * 128;
  const size_t stage_bytes = band_stage_bytes<T>(s.slot);
  const size_t pop_bytes = ((size_t)Q * s.slot * sizeof(T) + 127) / 128 * 128;
  auto stage_pop = [&](int j) {
    return reinterpret_cast<T*>(stages + (j % kBandStages) * stage_bytes);
  };
  auto stage_info = [&](int j) {
    return reinterpret_cast<uint2*>(stages + (j % kBandStages) * stage_bytes +
                                    pop_bytes);
  };

  const int band = blockIdx.x % s.nb, chunk = blockIdx.x / s.nb;
  const int y0 = (int)((long long)band * g.ly / s.nb);
  const int y1 = (int)((long long)(band + 1) * g.ly / s.nb);
  const int z0 = (int)((long long)chunk * g.lz / s.nc);
  const int z1 = (int)((long long)(chunk + 1) * g.lz / s.nc);
  const int nplanes = z1 - z0;
  // even chunks march up the planes, odd ones down
  const int dir = (chunk & 1) ? -1 : 1;
  const int zfirst = dir > 0 ? z0 : z1 - 1;  // first plane updated
  // march plane j (0 .. nplanes + 1) is lattice plane zw(j)
  auto plane_of = [&](int j) {
    const int zz = zfirst + (j - 1) * dir;
    return zz < 0 ? zz + g.lz : (zz >= g.lz ? zz - g.lz : zz);
  };
  const int rows = y1 - y0;
  const float shift = p.rho_shift;

  if (threadIdx.x == 0) {
    for (int k = 0; k < kBandStages; ++k) {
      mbar_init(&stage_full[k], 1);
      mbar_init(&stage_free[k], kBandD + kBandU);
    }
    for (int k = 0; k < kBandSlots; ++k) {
      mbar_init(&psi_full[k], kBandD);
      mbar_init(&psi_free[k], kBandU);
    }
    mbar_init(never, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x < kBandP) {
    // ---- producer: stage plane j once the stage's previous plane is done --
    if (threadIdx.x != 0) return;
    int issued = 0;
    bool ok = true;
    for (int j = 0; j < nplanes + 2 && ok; ++j) {
      const int k = j % kBandStages;
      if (j >= kBandStages &&
          !band_wait(&stage_free[k], (unsigned)((j / kBandStages - 1) & 1),
                     wait_ns, err)) {
        ok = false;
        break;
      }
      // the consumers' reads of this stage come before the copies rewrite it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const BandRanges r = band_ranges<T>(wtab, g, plane_of(j), y0, y1);
      unsigned bytes = 0;
      for (int q = 0; q < r.n; ++q)
        bytes += (unsigned)r.len[q] * (unsigned)(Q * sizeof(T) + sizeof(uint2));
      mbar_expect_tx(&stage_full[k], bytes);
      T* pop = stage_pop(j);
      uint2* info = stage_info(j);
      for (int q = 0; q < r.n; ++q) {
        const unsigned pb = (unsigned)(r.len[q] * sizeof(T));
        for (int i = 0; i < Q; ++i)
          bulk_copy(pop + i * s.slot + r.off[q], A + (size_t)i * cs + r.a[q], pb,
                    &stage_full[k]);
        bulk_copy(info + r.off[q], cinfo + r.a[q],
                  (unsigned)(r.len[q] * sizeof(uint2)), &stage_full[k]);
      }
      issued = j + 1;
    }
    if (!ok) {
      // leave no copy in flight: wait for the stages last issued
      for (int j = issued - 1; j >= 0 && j >= issued - kBandStages; --j)
        band_wait(&stage_full[j % kBandStages], (unsigned)((j / kBandStages) & 1),
                  wait_ns, err);
    }
    return;
  }

  if (threadIdx.x < kBandP + kBandD) {
    // ---- density warps: psi of the staged rows of march plane j -------------
    const int td = threadIdx.x - kBandP;
    for (int j = 0; j < nplanes + 2; ++j) {
      const int k = j % kBandSlots;
      if (j >= kBandSlots &&
          !band_wait(&psi_free[k], (unsigned)((j / kBandSlots - 1) & 1), wait_ns, err))
        return;
      if (!band_wait(&stage_full[j % kBandStages], (unsigned)((j / kBandStages) & 1),
                     wait_ns, err))
        return;
      const int zw = plane_of(j);
      const BandRanges r = band_ranges<T>(wtab, g, zw, y0, y1);
      const T* pop = stage_pop(j);
      const uint2* info = stage_info(j);
      float* slot = sp + k * SE;
      for (int q = 0; q < r.n; ++q) {
        const int kf = r.kf[q], ke = r.ke[q];
        for (int t = (kf & ~1) + 2 * td; t < ke; t += 2 * kBandD) {
          const int idx = r.off[q] + (t - r.a[q]);
          const BandNode na = band_node(info[idx]);
          const BandNode nbn = band_node(info[idx + 1]);
          const bool va = t >= kf && (na.nb & NB_SELF);
          const bool vb = t + 1 < ke && (nbn.nb & NB_SELF);
          if (!va && !vb) continue;
          float2 f[Q];
          stage_gather<T>(pop, s.slot, idx, shift, f);
          float2 d = p_dup(0.f);
#pragma unroll
          for (int i = 0; i < Q; ++i) d = p_add(d, f[i]);
          d.x = na.kind ? slab_density(p, na.kind) : inject_on(p, g, a, inj, na.y, d.x);
          d.y = nbn.kind ? slab_density(p, nbn.kind) : inject_on(p, g, a, inj, nbn.y, d.y);
          // a row's shared-memory rows: jr = y - (y0 - 1) (mod ly), and
          // jr + ly when the band wraps onto itself
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
      band_arrive(&psi_full[k]);
      band_arrive(&stage_free[j % kBandStages]);
    }
    return;
  }

  // ---- update warps: update u of the march needs march planes u, u+1, u+2 --
  const int tu = threadIdx.x - kBandP - kBandD;
  const float psi_solid = psi_of<float>(p, p.rhos);
  band_arrive(&stage_free[0]);  // march plane 0 is a halo plane
  if (stall && blockIdx.x == 0 && !band_wait(never, 0u, wait_ns, err)) return;
  for (int u = 0; u < nplanes; ++u) {
    for (int j = u == 0 ? 0 : u + 2; j <= u + 2; ++j)
      if (!band_wait(&psi_full[j % kBandSlots], (unsigned)((j / kBandSlots) & 1),
                     wait_ns, err))
        return;
    const int j = u + 1;
    if (!band_wait(&stage_full[j % kBandStages], (unsigned)((j / kBandStages) & 1),
                   wait_ns, err))
      return;
    const int z = zfirst + u * dir;
    const float* s0 = sp + ((u + 1) % kBandSlots) * SE;
    const float* sm = sp + ((dir > 0 ? u : u + 2) % kBandSlots) * SE;   // z - 1
    const float* spl = sp + ((dir > 0 ? u + 2 : u) % kBandSlots) * SE;  // z + 1
    // the own rows lie in the first staged range
    const BandRanges r = band_ranges<T>(wtab, g, z, y0, y1);
    const T* pop = stage_pop(j);
    const uint2* info = stage_info(j);
    const int kf = band_row_start(wtab, g, z, y0);
    const int ke = band_row_start(wtab, g, z, y1);
    for (int t = (kf & ~1) + 2 * tu; t < ke; t += 2 * kBandU) {
      const int idx = t - r.a[0];
      BandNode na = band_node(info[idx]);
      BandNode nbn = band_node(info[idx + 1]);
      const bool va = t >= kf && (na.nb & NB_SELF);
      const bool vb = t + 1 < ke && (nbn.nb & NB_SELF);
      if (!va && !vb) continue;
      float2 f[Q];
      stage_gather<T>(pop, s.slot, idx, shift, f);
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
              const float pa = ((na.nb >> opp(i)) & 1u) ? pl[ca + o] : psi_solid;
              const float pb = ((nbn.nb >> opp(i)) & 1u) ? pl[cb + o] : psi_solid;
              return make_float2(pa, pb);
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
    band_arrive(&psi_free[u % kBandSlots]);
    band_arrive(&stage_free[j % kBandStages]);
  }
  band_arrive(&stage_free[(nplanes + 1) % kBandStages]);  // the last halo plane
}

}  // namespace mlbm
