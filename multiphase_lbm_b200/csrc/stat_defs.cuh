// stat_defs.cuh -- the phase statistics record shared by the separate
// statistics pass (io_kernels.cuh) and the update pass that gathers them
// (stats_tap.cuh).
//
// Per node of the fluid: counts (fluid, liquid, vapour, liquid-solid and
// liquid-vapour boundary nodes), FP64 sums (mass, liquid/vapour pressure and
// density) and min/max of rho and p.  calc_cluster, src/multiphase_lbm.cu:
// 240-316; write_stats, :1061-1072.  Min and max start from the reference's
// 1e9 and -1e-9 (:1058-1059).
#pragma once

namespace mlbm {

enum { ST_NF, ST_NL, ST_NV, ST_NLS, ST_NLV, ST_MASS, ST_PL, ST_PV, ST_RL,
       ST_RV, ST_MINR, ST_MAXR, ST_MINP, ST_MAXP, ST_COUNT };

constexpr int kStatThreads = 256;  // blockDim (32, 8)
constexpr int kStatZ = 16;         // planes per block

__device__ __forceinline__ double stat_op(int k, double v, double o) {
  return (k == ST_MINR || k == ST_MINP) ? fmin(v, o)
         : (k == ST_MAXR || k == ST_MAXP) ? fmax(v, o)
                                           : v + o;
}
__device__ __forceinline__ double stat_identity(int k) {
  return (k == ST_MINR || k == ST_MINP) ? 1e9
         : (k == ST_MAXR || k == ST_MAXP) ? -1e-9
                                           : 0.0;
}

}  // namespace mlbm
