// compact.cuh -- the single-pass time step over a fluid-only ("compact
// rows") population layout.
//
// Layout.  Fluid nodes are numbered in (z, y, x) order; population i of the
// fluid node numbered k lives at cpop[i * cs + k].  Solid nodes own no
// storage, so DRAM moves 19 reads and 19 writes per fluid node and nothing
// for solids.  The index of a fluid node is found from the one-bit-per-node
// mask: wbase[r * wpr + w] is the number of fluid nodes before word w of row
// r = z * ly + y, so k(x, y, z) = wbase[r * wpr + x / 32] +
// popc(mask word & bits below x).  wbase has one extra entry at the end
// (the fluid node count), so wbase[r * wpr + wpr] is the end of row r.
//
// The AA pattern and the slot conventions are those of kernels.cuh, with the
// compact index in place of the dense node index.
//
// One launch per lattice step, no second pass over the populations.  The
// Shan-Chen force at step t+1 needs psi(rho) of every neighbour, and rho(m,
// t+1) = sum_i f*_i(m - e_i, t) (with halfway bounce-back) is a sum of
// post-collision populations of step t.  Each block of step t owns a tile of
// rows [y0, y1) x planes [z0, z1) (full rows in x) and, while it collides its
// nodes, accumulates the part of rho(t+1) that its own outputs contribute to
// every target node in the tile and its one-node halo.  The accumulation is
// an integer (fixed-point, 2^-40) sum in shared memory, so it does not depend
// on the order of the additions and the result is deterministic.  There are
// two sets of part buffers: a step reads the set its predecessor wrote and
// writes the other, so no block reads a part that another block of the same
// launch is rewriting.  Each sum is written once to part[s][k] of the set:
//   s = 0: the target is one of this tile's own nodes;
//   s = 1: the target is in the neighbouring tile in y (same z chunk);
//   s = 2: the target is in the neighbouring chunk in z (same y tile);
//   s = 3: the target is in the diagonal (y and z) neighbour.
// At step t+1 the block that needs psi of node m (its own nodes and its
// halo) adds the parts that exist for m: part 0 always, part 1 if m is in
// the first or last row of its y tile, part 2 if in the first or last plane
// of its z chunk, part 3 if both.  Every part is written by exactly one
// block (the tiles have at least two rows and planes and there are at least
// two tiles along y and z), and only the kernel boundary orders writer and
// reader, so no block waits for another.
//
// rho used in the collision of a node is the sum of its 19 gathered
// populations in the order i = 0..18, bit for bit the two-pass value; psi
// of the neighbours comes from the parts, which agree with the two-pass rho
// to a few units in the last place (different summation).
//
// Within a block the tile is walked plane by plane along z.  Shared memory
// holds (W = rows + 2):
//   psiw  [3][W][lx + 2]  psi of planes z-1, z, z+1 (x halo columns at 0 and
//                         lx+1, periodic copies);
//   acc   [3][W][lx]      fixed-point part sums of planes z-1, z, z+1;
//   rinfo [4][W][2 wpr + 1] mask words and wbase entries of planes
//                         z-1 .. z+2 (rows y0-1 .. y1);
//   xlist [rows * lx]     (row << 16 | x) of the fluid nodes of plane z, in
//                         compact order.
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

// Tiling and buffers of the compact layout (device pointers).
struct CArgs {
  const uint32_t* mask;   // [rows][wpr]
  const uint32_t* wbase;  // [rows * wpr + 1]
  const int* ytab;        // [ly]: tile | first-row bit 24 | last-row bit 25
  const int* ztab;        // [lz]: chunk | first-plane bit 24 | last-plane bit 25
  const int* ystart;      // [nty + 1]
  const int* zstart;      // [nzc + 1]
  const float* part_rd;   // [4][cs] parts written by the previous step
  float* part_wr;         // [4][cs] parts of the next step
  long long cs;           // compact plane stride (elements)
  int nty, nzc;
  int rows_max;           // largest tile height (shared-memory sizing)
};

constexpr int kEdgeLo = 1 << 24, kEdgeHi = 1 << 25, kTileMask = (1 << 24) - 1;
constexpr float kFix = 1099511627776.0f;        // 2^40
constexpr float kUnfix = 9.094947017729282e-13f;  // 2^-40

__host__ __device__ constexpr int c_wcols(int lx) { return lx + 2; }
__host__ __device__ constexpr int c_rwords(int wpr) { return 2 * wpr + 1; }

// Shared-memory bytes of k_compact_step for a tile height and row length.
__host__ __device__ inline size_t compact_smem_bytes(int rows_max, int lx,
                                                     int wpr) {
  const size_t W = rows_max + 2;
  return 3 * W * lx * 8                      // acc (int64)
         + 3 * W * c_wcols(lx) * 4           // psiw
         + 4 * W * c_rwords(wpr) * 4         // rinfo
         + (size_t)rows_max * lx * 4;        // xlist
}

__device__ __forceinline__ uint32_t low_bits(int x) {
  return (x & 31) ? (0xffffffffu >> (32 - (x & 31))) : 0u;
}

// Compact index of node (x, y, z) from the global tables (the node must be
// fluid).
__device__ __forceinline__ long long compact_index(const CArgs& c,
                                                   const Geom& g, int x, int y,
                                                   int z) {
  const long long r = (long long)z * g.ly + y;
  const uint32_t w = __ldg(c.mask + r * g.wpr + (x >> 5));
  return (long long)__ldg(c.wbase + r * g.wpr + (x >> 5)) +
         __popc(w & low_bits(x));
}

// Per-word fluid counts of every mask row (the host scans them into wbase).
static __global__ void k_word_counts(const uint32_t* __restrict__ mask,
                                     uint32_t* __restrict__ counts,
                                     long long nwords) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nwords) counts[i] = __popc(mask[i]);
}

// Dense <-> compact copies of the populations (all slots of fluid nodes).
template <typename T, bool TO_COMPACT>
__global__ void k_convert(T* __restrict__ dense, T* __restrict__ cpop,
                          CArgs c, Geom g) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(c.mask, g, x, y, z)) return;
  const long long n = node_index(g, x, y, z);
  const long long k = compact_index(c, g, x, y, z);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if (TO_COMPACT)
      cpop[i * c.cs + k] = dense[i * g.plane + n];
    else
      dense[i * g.plane + n] = cpop[i * c.cs + k];
  }
}

// part[0][k] of the set the next step reads = rho of fluid node k in the
// current (dense) state, the raw sum of its 19 stored populations; parts
// 1..3 of that set are cleared by the caller.
template <typename T, int PHASE>
__global__ void k_seed_parts(const T* __restrict__ pop,
                             const uint32_t* __restrict__ nbw, CArgs c, Geom g,
                             Phys p) {
  using R = typename Pop<T>::Real;
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  const int n = (int)node_index(g, x, y, z);
  const uint32_t nb = nbw[n];
  if (!(nb & NB_SELF)) return;
  Nbr a;
  a.init(g, x, y, z);
  R f[Q];
  gather<T, PHASE>(pop, g.plane, a, nb, n, R(p.rho_shift), f);
  R d = R(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
  c.part_wr[compact_index(c, g, x, y, z)] = (float)d;
}

// Value the next step reads back for a stored population.
template <typename T>
__device__ __forceinline__ float stored_value(float v, float s) {
  return v;
}
template <>
__device__ __forceinline__ float stored_value<__half>(float v, float s) {
  return __half2float(__float2half_rn(v - s)) + s;
}

template <typename T, int PHASE, int OUT>
__global__ void __launch_bounds__(256, 2)
    k_compact_step(T* __restrict__ cpop, CArgs c, float* __restrict__ rho_out,
                   float* __restrict__ psi_out, float* __restrict__ vel,
                   Geom g, Phys p, StepArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int lx = g.lx, wpr = g.wpr, wc = c_wcols(lx), rw = c_rwords(wpr);
  const int W = c.rows_max + 2;
  long long* acc = reinterpret_cast<long long*>(smem_raw);
  float* psiw = reinterpret_cast<float*>(acc + 3 * W * lx);
  uint32_t* rinfo = reinterpret_cast<uint32_t*>(psiw + 3 * W * wc);
  uint32_t* xlist = rinfo + 4 * W * rw;

  const int ty = blockIdx.x % c.nty, tz = blockIdx.x / c.nty;
  const int y0 = c.ystart[ty], y1 = c.ystart[ty + 1];
  const int z0 = c.zstart[tz], z1 = c.zstart[tz + 1];
  const int rows = y1 - y0, Wt = rows + 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  const float shift = p.rho_shift;
  const float psi_solid = psi_of<float>(p, p.rhos);
  const float psi_in = psi_of<float>(p, p.rho_inlet);
  const float psi_out_slab = psi_of<float>(p, p.rho_outlet);

  auto wrapz = [&](int q) { return q < 0 ? q + g.lz : (q >= g.lz ? q - g.lz : q); };
  auto wrapy = [&](int v) { return v < 0 ? v + g.ly : (v >= g.ly ? v - g.ly : v); };
  auto ring3 = [&](int q) { return (q - z0 + 1) % 3; };
  auto ring4 = [&](int q) { return (q - z0 + 1) & 3; };
  // rinfo of plane q, window row j: mask words, then wbase entries
  auto rmask = [&](int q, int j) { return rinfo + (ring4(q) * W + j) * rw; };
  auto rbase = [&](int q, int j) { return rinfo + (ring4(q) * W + j) * rw + wpr; };

  auto load_rinfo = [&](int q) {
    const int zq = wrapz(q);
    for (int e = tid; e < Wt * rw; e += nt) {
      const int j = e / rw, w = e - j * rw;
      const long long r = (long long)zq * g.ly + wrapy(y0 - 1 + j);
      rmask(q, j)[w] = w < wpr ? __ldg(c.mask + r * wpr + w)
                               : __ldg(c.wbase + r * wpr + (w - wpr));
    }
  };
  // psi of plane q (all window rows) from the parts of the previous step
  auto fill_psi = [&](int q) {
    const int zq = wrapz(q);
    const int zt = __ldg(c.ztab + zq);
    const bool zedge = (zt & (kEdgeLo | kEdgeHi)) != 0;
    float* dst = psiw + ring3(q) * W * wc;
    for (int e = tid; e < Wt * lx; e += nt) {
      const int j = e / lx, x = e - j * lx;
      const int y = wrapy(y0 - 1 + j);
      const uint32_t mw = rmask(q, j)[x >> 5];
      float v;
      if (!((mw >> (x & 31)) & 1u)) {
        v = psi_solid;
      } else {
        const int kind = bc_kind(p, g, x);
        if (kind) {
          v = kind == 1 ? psi_in : psi_out_slab;
        } else {
          const long long k = (long long)rbase(q, j)[x >> 5] + __popc(mw & low_bits(x));
          const bool yedge = (__ldg(c.ytab + y) & (kEdgeLo | kEdgeHi)) != 0;
          float d = __ldcg(c.part_rd + k);
          if (yedge) d = radd(d, __ldcg(c.part_rd + c.cs + k));
          if (zedge) d = radd(d, __ldcg(c.part_rd + 2 * c.cs + k));
          if (yedge && zedge) d = radd(d, __ldcg(c.part_rd + 3 * c.cs + k));
          v = psi_of<float>(p, inject<float>(p, g, a, y, d));
        }
      }
      float* row = dst + j * wc;
      row[x + 1] = v;
      if (x == 0) row[lx + 1] = v;
      if (x == lx - 1) row[0] = v;
    }
  };
  // write the finished part sums of plane q and clear their slot
  auto flush = [&](int q) {
    const int zq = wrapz(q);
    const int zt = __ldg(c.ztab + zq) & kTileMask;
    long long* src = acc + ring3(q) * W * lx;
    for (int e = tid; e < Wt * lx; e += nt) {
      const int j = e / lx, x = e - j * lx;
      const uint32_t mw = rmask(q, j)[x >> 5];
      const long long v = src[j * lx + x];
      src[j * lx + x] = 0;
      if (!((mw >> (x & 31)) & 1u)) continue;
      const int y = wrapy(y0 - 1 + j);
      const int s = ((__ldg(c.ytab + y) & kTileMask) != ty ? 1 : 0) + (zt != tz ? 2 : 0);
      const long long k = (long long)rbase(q, j)[x >> 5] + __popc(mw & low_bits(x));
      c.part_wr[s * c.cs + k] = __ll2float_rn(v) * kUnfix;
    }
  };

  for (int e = tid; e < 3 * W * lx; e += nt) acc[e] = 0;
  load_rinfo(z0 - 1);
  load_rinfo(z0);
  __syncthreads();
  fill_psi(z0 - 1);
  fill_psi(z0);

  for (int z = z0; z < z1; ++z) {
    load_rinfo(z + 1);
    __syncthreads();
    fill_psi(z + 1);
    // fluid nodes of plane z, rows y0..y1-1 (one contiguous compact range)
    const long long kb = rbase(z, 1)[0];
    const long long ke = rbase(z, rows)[wpr];
    for (int e = tid; e < rows * lx; e += nt) {
      const int jr = e / lx, x = e - jr * lx;
      const uint32_t mw = rmask(z, jr + 1)[x >> 5];
      if ((mw >> (x & 31)) & 1u) {
        const long long k = (long long)rbase(z, jr + 1)[x >> 5] + __popc(mw & low_bits(x));
        xlist[k - kb] = ((uint32_t)jr << 16) | (uint32_t)x;
      }
    }
    __syncthreads();

    // ---- update the fluid nodes of plane z ------------------------------
    const float* pm = psiw + ring3(z - 1) * W * wc;
    const float* p0 = psiw + ring3(z) * W * wc;
    const float* pp = psiw + ring3(z + 1) * W * wc;
    long long* am = acc + ring3(z - 1) * W * lx;
    long long* a0 = acc + ring3(z) * W * lx;
    long long* ap = acc + ring3(z + 1) * W * lx;
    const int zg = z >= g.lz ? z - g.lz : z;
    for (long long k = kb + tid; k < ke; k += nt) {
      const uint32_t xl = xlist[k - kb];
      const int jr = (int)(xl >> 16), x = (int)(xl & 0xffff);
      const int y = y0 + jr;
      const int jw = jr + 1;  // window row
      // fluid flags and compact indices of the 18 neighbours x + e_i
      uint32_t nbf = 0;
      int nk[Q];
#pragma unroll
      for (int i = 1; i < Q; ++i) {
        const int q = z + ez(i);
        const int jj = jw + ey(i);
        int xx = x + ex(i);
        xx = xx < 0 ? xx + lx : (xx >= lx ? xx - lx : xx);
        const uint32_t mw = rmask(q, jj)[xx >> 5];
        const bool fl = (mw >> (xx & 31)) & 1u;
        nbf |= (uint32_t)fl << i;
        nk[i] = PHASE == 0 ? (int)(rbase(q, jj)[xx >> 5] + __popc(mw & low_bits(xx))) : 0;
      }
      nk[0] = (int)k;
      const int kind = bc_kind(p, g, x);
      float f[Q];
      float d = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
      if (kind) {
        d = slab_density(p, kind);
        slab_populations<float>(d, f);
      } else {
        // gather: f_i(x) = f*_i(x - e_i) from slot opp(i) of x - e_i (phase 0)
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const float s = shift * weight<float>(i);
          long long src = k;
          int slot = i;
          if (PHASE == 0 && i != 0 && ((nbf >> opp(i)) & 1u)) {
            src = nk[opp(i)];
            slot = opp(i);
          }
          f[i] = Pop<T>::ld(cpop + slot * c.cs + src, s);
        }
        d = sum_density<float>(p, g, a, y, f);
        const int cxy = jw * wc + x + 1;
        collide<float>(
            p, d, p0[cxy],
            [&](int i) {
              const float* pl = ez(i) < 0 ? pm : (ez(i) > 0 ? pp : p0);
              return pl[cxy + ey(i) * wc + ex(i)];
            },
            f, ux, uy, uz);
      }
      if (OUT & OUT_RHO) {
        const long long n = node_index(g, x, y, zg);
        rho_out[n] = d;
        store_psi<float>(psi_out, g, x, y, zg, psi_of<float>(p, d));
      }
      if (OUT & OUT_VEL) {
        const long long n = node_index(g, x, y, zg);
        vel[3 * n] = ux;
        vel[3 * n + 1] = uy;
        vel[3 * n + 2] = uz;
      }
      // store, and add each population to the part sum of the node that
      // reads it next step: x + e_i if fluid, else x itself (bounce-back)
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const float s = shift * weight<float>(i);
        const bool to_nb = i != 0 && ((nbf >> i) & 1u);
        long long dst = k;
        int slot = opp(i);
        if (PHASE == 0 && to_nb) {
          dst = nk[i];
          slot = i;
        }
        Pop<T>::st(cpop + slot * c.cs + dst, f[i], s);
        const long long fx = __float2ll_rn(stored_value<T>(f[i], s) * kFix);
        long long* cell;
        if (to_nb) {
          int xx = x + ex(i);
          xx = xx < 0 ? xx + lx : (xx >= lx ? xx - lx : xx);
          long long* pl = ez(i) < 0 ? am : (ez(i) > 0 ? ap : a0);
          cell = pl + (jw + ey(i)) * lx + xx;
        } else {
          cell = a0 + jw * lx + x;
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(cell),
                  (unsigned long long)fx);
      }
    }
    __syncthreads();
    flush(z - 1);
  }
  __syncthreads();
  flush(z1 - 1);
  flush(z1);
}

}  // namespace mlbm
