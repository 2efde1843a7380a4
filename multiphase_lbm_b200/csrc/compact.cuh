// compact.cuh -- the single-pass time step over a fluid-only ("compact
// rows") population layout.
//
// Layout.  Fluid nodes are numbered in (z, y, x) order; population i of the
// fluid node numbered k lives at cpop[i * cs + k].  Solid nodes own no
// storage, so DRAM moves 19 reads and 19 writes per fluid node and nothing
// for solids.  The index of a fluid node is found from the one-bit-per-node
// mask: wbase[r * wpr + w] is the compact index of the first fluid node at
// or after word w of row r = z * ly + y, so k(x, y, z) = wbase[r * wpr +
// x / 32] + popc(mask word & bits below x).  A plane with an odd fluid count
// is followed by one unused slot (a hole), so every plane starts at an even
// index; the end of row r is therefore wbase + popc of its last word (not
// always the next row's start).  wbase has one extra entry at the end (the
// slot count).
// cnb[k] is the neighbour word of node k (kernels.cuh: bit 0 fluid, bit i
// the pull source x - e_i fluid, bits 19-20 the drainage slab kind).
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
// Within a block the tile is walked plane by plane along z with one barrier
// per plane: the phase of plane z updates plane z and, on the side, fills
// psi of plane z+2, lists the fluid nodes of plane z+1, writes the finished
// part sums of plane z-2 and loads the row tables of plane z+3.  Shared
// memory (W = rows + 2 window rows y0-1 .. y1, P = wpr + 1):
//   acc   [4][W][lx]     fixed-point part sums of planes z-2 .. z+1;
//   rows  [6][W][P]      (mask word, wbase) pairs of planes z-2 .. z+3, the
//                        last pair of a row holding (0, end of row);
//   psiw  [4][W][lx + 2] psi of planes z-1 .. z+2 (x halo columns 0, lx+1);
//   xlist [2][rows * lx] (row << 16 | x) of the fluid nodes of planes z and
//                        z+1 in compact order.
// Loops over window positions give each warp one mask word (32 x positions)
// of one row at a time: lane = bit, rank = wbase + popc(mask & lanes below).
#pragma once

#include "kernels.cuh"
#include "lattice.cuh"

namespace mlbm {

// Tiling and buffers of the compact layout (device pointers).
struct CArgs {
  const uint32_t* mask;   // [rows][wpr]
  const uint32_t* wbase;  // [rows * wpr + 1]
  const uint32_t* cnb;    // [nfluid] neighbour words in compact order
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
constexpr int kCompactThreads = 256;

// Shared-memory bytes of k_compact_step for a tile height and row length.
__host__ __device__ inline size_t compact_smem_bytes(int rows_max, int lx,
                                                     int wpr) {
  const size_t W = rows_max + 2;
  return 4 * W * lx * 8                      // acc (int64)
         + 6 * W * (wpr + 1) * 8             // row pairs
         + 4 * W * (lx + 2) * 4              // psiw
         + 2 * (size_t)rows_max * lx * 4;    // xlist
}

__device__ __forceinline__ uint32_t low_bits(int x) {
  return (1u << (x & 31)) - 1u;
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

// Dense <-> compact copies of the populations (all slots of fluid nodes);
// the copy to the compact layout also takes the neighbour words.
template <typename T, bool TO_COMPACT>
__global__ void k_convert(T* __restrict__ dense, T* __restrict__ cpop,
                          const uint32_t* __restrict__ nbw,
                          uint32_t* __restrict__ cnb, CArgs c, Geom g) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.lx || y >= g.ly) return;
  if (!fluid_at(c.mask, g, x, y, z)) return;
  const long long n = node_index(g, x, y, z);
  const long long k = compact_index(c, g, x, y, z);
  if (TO_COMPACT) cnb[k] = nbw[n];
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
__device__ __forceinline__ float stored_value(float v, float) {
  return v;
}
template <>
__device__ __forceinline__ float stored_value<__half>(float v, float s) {
  return __fadd_rn(__half2float(__float2half_rn(__fsub_rn(v, s))), s);
}

// The density injection of compute_density (include/iteration_device.cuh:
// 46-59) with its step test, the same for every node of a launch, hoisted
// out: `on` is that test.
__device__ __forceinline__ float inject_on(const Phys& p, const Geom& g,
                                           const StepArgs& s, bool on, int y,
                                           float d) {
  if (!on || !((float)y < p.inject_position * (float)g.ly)) return d;
  const float inc = rmul(p.rho_increment, (float)s.reverse);
  switch (s.inject_type) {
    case 0: return radd(d, inc);
    case 1: return d < p.rhol_spinodal ? radd(d, inc) : d;
    case 2: return d > p.rhol_spinodal ? radd(d, inc) : d;
    default: return d;
  }
}

template <typename T, int PHASE, int OUT>
__global__ void __launch_bounds__(kCompactThreads, 2)
    k_compact_step(T* __restrict__ cpop, CArgs c, float* __restrict__ rho_out,
                   float* __restrict__ psi_out, float* __restrict__ vel,
                   Geom g, Phys p, StepArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int lx = g.lx, wpr = g.wpr, wc = lx + 2, P = wpr + 1;
  const int W = c.rows_max + 2;
  long long* acc = reinterpret_cast<long long*>(smem_raw);
  uint2* rp = reinterpret_cast<uint2*>(acc + 4 * W * lx);
  float* psiw = reinterpret_cast<float*>(rp + 6 * W * P);
  uint32_t* xlist = reinterpret_cast<uint32_t*>(psiw + 4 * W * wc);
  const int xl_stride = c.rows_max * lx;

  const int ty = blockIdx.x % c.nty, tz = blockIdx.x / c.nty;
  const int y0 = c.ystart[ty], y1 = c.ystart[ty + 1];
  const int z0 = c.zstart[tz], z1 = c.zstart[tz + 1];
  const int rows = y1 - y0, Wt = rows + 2;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = kCompactThreads / 32;
  const uint32_t lanes_below = (1u << lane) - 1u;
  const float shift = p.rho_shift;
  const float psi_solid = psi_of<float>(p, p.rhos);
  const float psi_in = psi_of<float>(p, p.rho_inlet);
  const float psi_out_slab = psi_of<float>(p, p.rho_outlet);
  const bool inj = p.rho_inject_period != 0ull &&
                   (unsigned long long)a.step % p.rho_inject_period == 0ull;

  auto wrapz = [&](int q) { return q < 0 ? q + g.lz : (q >= g.lz ? q - g.lz : q); };
  auto wrapy = [&](int v) { return v < 0 ? v + g.ly : (v >= g.ly ? v - g.ly : v); };
  // ring slots of plane q (q >= z0 - 2)
  auto r4 = [&](int q) { return (q - z0 + 2) & 3; };
  auto r6 = [&](int q) { return (q - z0 + 2) % 6; };
  auto rows_of = [&](int q) { return rp + r6(q) * W * P; };

  auto load_rows = [&](int q) {
    const int zq = wrapz(q);
    uint2* dst = rows_of(q);
    for (int e = tid; e < Wt * P; e += kCompactThreads) {
      const int j = e / P, w = e - j * P;
      const long long r = (long long)zq * g.ly + wrapy(y0 - 1 + j);
      uint2 v;
      if (w < wpr) {
        v.x = __ldg(c.mask + r * wpr + w);
        v.y = __ldg(c.wbase + r * wpr + w);
      } else {  // (0, end of row)
        v.x = 0u;
        v.y = __ldg(c.wbase + r * wpr + wpr - 1) +
              __popc(__ldg(c.mask + r * wpr + wpr - 1));
      }
      dst[j * P + w] = v;
    }
  };
  // psi of plane q (all window rows) from the parts of the previous step;
  // one warp per (row, mask word)
  auto fill_psi = [&](int q) {
    const int zq = wrapz(q);
    const bool zedge = (__ldg(c.ztab + zq) & (kEdgeLo | kEdgeHi)) != 0;
    float* dst = psiw + r4(q) * W * wc;
    const uint2* rq = rows_of(q);
    for (int u = warp; u < Wt * wpr; u += nwarps) {
      const int j = u / wpr, w = u - j * wpr;
      const int x = w * 32 + lane;
      if (x >= lx) continue;
      const uint2 mw = rq[j * P + w];
      float v = psi_solid;
      if ((mw.x >> lane) & 1u) {
        const int kind = bc_kind(p, g, x);
        if (kind) {
          v = kind == 1 ? psi_in : psi_out_slab;
        } else {
          const int y = wrapy(y0 - 1 + j);
          const bool yedge = (__ldg(c.ytab + y) & (kEdgeLo | kEdgeHi)) != 0;
          const long long k = (long long)mw.y + __popc(mw.x & lanes_below);
          float d = __ldcg(c.part_rd + k);
          if (yedge) d = radd(d, __ldcg(c.part_rd + c.cs + k));
          if (zedge) d = radd(d, __ldcg(c.part_rd + 2 * c.cs + k));
          if (yedge && zedge) d = radd(d, __ldcg(c.part_rd + 3 * c.cs + k));
          v = psi_of<float>(p, inject_on(p, g, a, inj, y, d));
        }
      }
      float* row = dst + j * wc;
      row[x + 1] = v;
      if (x == 0) row[lx + 1] = v;
      if (x == lx - 1) row[0] = v;
    }
  };
  // (row << 16 | x) of the fluid nodes of plane q (own rows), by compact index
  auto list_nodes = [&](int q) {
    const uint2* rq = rows_of(q);
    uint32_t* xl = xlist + ((q - z0) & 1) * xl_stride;
    const uint32_t kb = rq[P].y;  // first node of row y0
    for (int u = warp; u < rows * wpr; u += nwarps) {
      const int jr = u / wpr, w = u - jr * wpr;
      const uint2 mw = rq[(jr + 1) * P + w];
      if ((mw.x >> lane) & 1u)
        xl[mw.y + __popc(mw.x & lanes_below) - kb] =
            ((uint32_t)jr << 16) | (uint32_t)(w * 32 + lane);
    }
  };
  // write the finished part sums of plane q and clear their slot
  auto flush = [&](int q) {
    const int zq = wrapz(q);
    const bool zo = (__ldg(c.ztab + zq) & kTileMask) != tz;
    long long* src = acc + r4(q) * W * lx;
    const uint2* rq = rows_of(q);
    for (int u = warp; u < Wt * wpr; u += nwarps) {
      const int j = u / wpr, w = u - j * wpr;
      const int x = w * 32 + lane;
      if (x >= lx) continue;
      const long long v = src[j * lx + x];
      src[j * lx + x] = 0;
      const uint2 mw = rq[j * P + w];
      if (!((mw.x >> lane) & 1u)) continue;
      const int y = wrapy(y0 - 1 + j);
      const int s = ((__ldg(c.ytab + y) & kTileMask) != ty ? 1 : 0) + (zo ? 2 : 0);
      const long long k = (long long)mw.y + __popc(mw.x & lanes_below);
      c.part_wr[s * c.cs + k] = __ll2float_rn(v) * kUnfix;
    }
  };

  // ---- prologue: psi of planes z0-1 .. z0+1, rows of planes .. z0+2 -------
  for (int e = tid; e < 4 * W * lx; e += kCompactThreads) acc[e] = 0;
  for (int q = z0 - 1; q <= z0 + 2 && q <= z1; ++q) load_rows(q);
  __syncthreads();
  for (int q = z0 - 1; q <= z0 + 1 && q <= z1; ++q) fill_psi(q);
  list_nodes(z0);
  __syncthreads();

  for (int z = z0; z < z1; ++z) {
    // ---- side work of this phase (touches no slot the update uses) --------
    if (z + 2 <= z1) fill_psi(z + 2);
    if (z + 1 < z1) list_nodes(z + 1);
    if (z - 2 >= z0 - 1) flush(z - 2);
    if (z + 3 <= z1) load_rows(z + 3);

    // ---- update the fluid nodes of plane z -------------------------------
    const uint2* rm = rows_of(z - 1);
    const uint2* r0 = rows_of(z);
    const uint2* rpz = rows_of(z + 1);
    const float* pm = psiw + r4(z - 1) * W * wc;
    const float* p0 = psiw + r4(z) * W * wc;
    const float* pp = psiw + r4(z + 1) * W * wc;
    long long* am = acc + r4(z - 1) * W * lx;
    long long* a0 = acc + r4(z) * W * lx;
    long long* ap = acc + r4(z + 1) * W * lx;
    const uint32_t* xl = xlist + ((z - z0) & 1) * xl_stride;
    const int kb = (int)r0[P].y;               // first node of row y0
    const int ke = (int)r0[rows * P + wpr].y;  // end of row y1-1
    for (int k = kb + tid; k < ke; k += kCompactThreads) {
      const uint32_t xe = xl[k - kb];
      const int jr = (int)(xe >> 16), x = (int)(xe & 0xffff);
      const int y = y0 + jr;
      const int jw = jr + 1;  // window row
      const uint32_t nb = __ldg(c.cnb + k);
      const int kind = nb_kind(nb);
      // compact index of x + e_i (used only where that node is fluid; phase
      // 0 only): the rank of x in each neighbour row, then x - 1 -> rank - 1
      // and x + 1 -> rank + fluid(x), with the periodic wrap in x
      int nk[Q];
      if (PHASE == 0) {
        const bool xlo = x == 0, xhi = x == lx - 1;
        const int w = x >> 5;
        const uint32_t lb = low_bits(x);
        auto row_rank = [&](const uint2* rr, int j, int& r_, int& rl, int& rh) {
          const uint2* row = rr + j * P;
          const uint2 v = row[w];
          r_ = (int)v.y + __popc(v.x & lb);
          rl = xlo ? (int)row[wpr].y - 1 : r_ - 1;
          rh = xhi ? (int)row[0].y : r_ + (int)((v.x >> (x & 31)) & 1u);
        };
        int r_, rl, rh;
        nk[1] = xlo ? (int)r0[jw * P + wpr].y - 1 : k - 1;  // (-1, 0, 0)
        nk[10] = xhi ? (int)r0[jw * P].y : k + 1;           // (+1, 0, 0)
        row_rank(r0, jw - 1, r_, rl, rh);  // row y-1
        nk[2] = r_; nk[4] = rl; nk[14] = rh;
        row_rank(r0, jw + 1, r_, rl, rh);  // row y+1
        nk[11] = r_; nk[5] = rl; nk[13] = rh;
        row_rank(rm, jw, r_, rl, rh);      // plane z-1
        nk[3] = r_; nk[6] = rl; nk[16] = rh;
        row_rank(rpz, jw, r_, rl, rh);     // plane z+1
        nk[12] = r_; nk[7] = rl; nk[15] = rh;
        row_rank(rm, jw - 1, r_, rl, rh);  nk[8] = r_;   // (0, -1, -1)
        row_rank(rpz, jw - 1, r_, rl, rh); nk[9] = r_;   // (0, -1, +1)
        row_rank(rpz, jw + 1, r_, rl, rh); nk[17] = r_;  // (0, +1, +1)
        row_rank(rm, jw + 1, r_, rl, rh);  nk[18] = r_;  // (0, +1, -1)
      }
      nk[0] = k;
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
          int src = k, slot = i;
          if (PHASE == 0 && i != 0 && ((nb >> i) & 1u)) {
            src = nk[opp(i)];
            slot = opp(i);
          }
          f[i] = Pop<T>::ld(cpop + slot * c.cs + src, s);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) d = radd(d, f[i]);
        d = inject_on(p, g, a, inj, y, d);
        const int cxy = jw * wc + x + 1;
        collide<float>(
            p, d, p0[cxy],
            [&](int i) {
              const float* pl = ez(i) < 0 ? pm : (ez(i) > 0 ? pp : p0);
              return pl[cxy + ey(i) * wc + ex(i)];
            },
            f, ux, uy, uz);
      }
      if (OUT & (OUT_RHO | OUT_VEL)) {
        const long long n = node_index(g, x, y, z);
        if (OUT & OUT_RHO) {
          rho_out[n] = d;
          store_psi<float>(psi_out, g, x, y, z, psi_of<float>(p, d));
        }
        if (OUT & OUT_VEL) {
          vel[3 * n] = ux;
          vel[3 * n + 1] = uy;
          vel[3 * n + 2] = uz;
        }
      }
      // store, and add each population to the part sum of the node that
      // reads it next step: x + e_i if fluid, else x itself (bounce-back)
      const int cell = jw * lx + x;
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const float s = shift * weight<float>(i);
        const bool to_nb = i != 0 && ((nb >> opp(i)) & 1u);
        int dst = k, slot = opp(i);
        if (PHASE == 0 && to_nb) {
          dst = nk[i];
          slot = i;
        }
        Pop<T>::st(cpop + slot * c.cs + dst, f[i], s);
        const long long fx = __float2ll_rn(stored_value<T>(f[i], s) * kFix);
        long long* t;
        if (to_nb) {
          long long* pl = ez(i) < 0 ? am : (ez(i) > 0 ? ap : a0);
          int off = cell + ey(i) * lx + ex(i);
          if (ex(i) < 0 && x == 0) off += lx;
          if (ex(i) > 0 && x == lx - 1) off -= lx;
          t = pl + off;
        } else {
          t = a0 + cell;
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(t),
                  (unsigned long long)fx);
      }
    }
    __syncthreads();
  }
  // ---- epilogue: the last three target planes ----------------------------
  for (int q = z1 - 2; q <= z1; ++q)
    if (q >= z0 - 1) flush(q);
}

}  // namespace mlbm
