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
// A block marches the chunk plane by plane.  For plane z + 1 it forms rho
// and psi of its rows plus one halo row on either side (y0 - 1 and y1,
// periodic) into a ring of four shared-memory psi planes; after one barrier
// it updates the own rows of plane z with psi of planes z - 1, z, z + 1 from
// shared memory.  The halo rows belong to the neighbouring bands, whose
// blocks read them at about the same time, and the update re-reads the rows
// the density phase has just loaded: both come from L2, so DRAM sees every
// population once per step (plus two planes per chunk at the chunk edges).
// Four ring slots let the density phase of the next plane overwrite the
// slot the update has finished with, with one barrier per plane.
//
// Per node the arithmetic is the two-pass kernels': rho summed in order
// i = 0..18 plus injection, psi_of, collide2 of pair.cuh (two nodes per
// thread in packed FP32), the drainage slabs' rest equilibrium.  Results are
// bit-identical to the two-pass kernels, whose step from phase 1 reads and
// writes the same values at other addresses.
//
// Neighbours that are solid contribute psi(rhos) (wall adhesion,
// include/iteration_device.cuh:69-152); their shared-memory entries are
// never written and never read (the node's neighbour word selects).
#pragma once

#include "compact2.cuh"

namespace mlbm {

constexpr int kBandThreads = 128;
constexpr int kBandSlots = 4;

// Shared memory of a block: kBandSlots planes of (hmax + 2) rows of
// (lx + 2) psi values (ghost columns at 0 and lx + 1).
__host__ __device__ inline size_t band_smem_bytes(int hmax, int lx) {
  return (size_t)kBandSlots * (hmax + 2) * (lx + 2) * sizeof(float);
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

struct BandShape {
  int nb, nc;  // bands along y, chunks along z
  int hmax;    // rows of the tallest band
};

template <typename T, bool WRITE_RHO, bool WRITE_U>
__global__ void __launch_bounds__(kBandThreads, 4)
    k_band(const T* __restrict__ A, T* __restrict__ B, uint32_t cs,
           const uint2* __restrict__ cinfo, const uint2* __restrict__ wtab,
           float* __restrict__ rho_out, float* __restrict__ vel, Geom g,
           Phys p, StepArgs a, bool inj, BandShape s) {
  extern __shared__ float sp[];
  const int band = blockIdx.x % s.nb, chunk = blockIdx.x / s.nb;
  const int y0 = (int)((long long)band * g.ly / s.nb);
  const int y1 = (int)((long long)(band + 1) * g.ly / s.nb);
  const int z0 = (int)((long long)chunk * g.lz / s.nc);
  const int z1 = (int)((long long)(chunk + 1) * g.lz / s.nc);
  const int P = g.lx + 2;               // psi row pitch in shared memory
  const int SE = (s.hmax + 2) * P;      // psi plane
  const int rows = y1 - y0;
  const float shift = p.rho_shift;
  const float psi_solid = psi_of<float>(p, p.rhos);
  // all rows when the band and its halo wrap onto themselves
  const bool all_rows = rows + 2 >= g.ly;

  // rho and psi of the band's rows and halo rows of plane zz (periodic) into
  // its ring slot
  auto density = [&](int zz) {
    const int zw = zz < 0 ? zz + g.lz : (zz >= g.lz ? zz - g.lz : zz);
    float* slot = sp + ((zz - z0 + 1) & (kBandSlots - 1)) * SE;
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
    for (int r = 0; r < nr; ++r) {
      const int kf = band_row_start(wtab, g, zw, ra[r]);
      const int ke = band_row_start(wtab, g, zw, rb[r]);
      for (int t = (kf & ~1) + 2 * (int)threadIdx.x; t < ke;
           t += 2 * kBandThreads) {
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
        // a row's shared-memory rows: j = y - (y0 - 1) (mod ly), and j + ly
        // when the band wraps onto itself
        auto put = [&](const BandNode& n, float v) {
          int j = n.y - y0 + 1;
          if (j < 0) j += g.ly;
          if (j >= g.ly) j -= g.ly;
          for (; j < rows + 2; j += g.ly) {
            float* row = slot + j * P;
            row[n.x + 1] = v;
            if (n.x == 0) row[g.lx + 1] = v;
            if (n.x == g.lx - 1) row[0] = v;
          }
        };
        if (va) put(na, psi_of<float>(p, d.x));
        if (vb) put(nbn, psi_of<float>(p, d.y));
      }
    }
  };

  // force, collision and push of the band's own rows of plane z
  auto update = [&](int z) {
    const float* sm = sp + ((z - z0) & (kBandSlots - 1)) * SE;      // z - 1
    const float* s0 = sp + ((z - z0 + 1) & (kBandSlots - 1)) * SE;  // z
    const float* spl = sp + ((z - z0 + 2) & (kBandSlots - 1)) * SE; // z + 1
    const int kf = band_row_start(wtab, g, z, y0);
    const int ke = band_row_start(wtab, g, z, y1);
    for (int t = (kf & ~1) + 2 * (int)threadIdx.x; t < ke;
         t += 2 * kBandThreads) {
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
  };

  density(z0 - 1);
  density(z0);
  for (int z = z0; z < z1; ++z) {
    density(z + 1);
    __syncthreads();
    update(z);
  }
}

}  // namespace mlbm
