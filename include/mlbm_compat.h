/*
 * mlbm_compat.h -- the reference's own host<->device entry points, with
 * their signatures, implemented by libmlbm on the B200 kernels.
 *
 * Amber1995/multiphase_LBM drives its GPU through three functions declared
 * at include/iteration_host.h:30-60 and defined at src/iteration_host.cu:
 * 16-81.  A reference driver that includes this header instead of
 * iteration_host.h and links libmlbm runs unchanged:
 *
 *   transfer_parameter(...)            include/iteration_host.h:30-41
 *       stores the parameters of the lattice to be created.
 *   multiphaselbm_initialization(...)  include/iteration_host.h:43-49
 *       creates the lattice on the current device, uploads *is_fluid and
 *       *rho (host or managed arrays [x][y][z]), initialises it, and writes
 *       the initial rho (solids = rhos) and pressure back into *rho and
 *       *pressure.  psi, collision_f, stream_f and force are not used: the
 *       populations live in libmlbm's own single AA lattice.
 *   multiphaselbm_iteration(step, statPeriod, reverse, inject_type)
 *       include/iteration_host.h:56-57
 *       advances one step; when step % statPeriod == 0 it copies rho and
 *       pressure back into the driver's arrays and waits for the copy, so
 *       the driver's statistics read fresh values (the reference reads its
 *       managed arrays without synchronising, src/multiphase_lbm.cu:595-600).
 *
 * The lattice size is a compile-time constant in the reference
 * (include/lbm_model.cuh:4-6).  When the including translation unit defines
 * the macros lx, ly and lz, transfer_parameter passes them on automatically; otherwise
 * call mlbm_compat_set_domain first (default 400^3).  These void functions
 * cannot return a status: on failure they print the error and exit, as the
 * reference's cudaErrorCheck does (include/iteration_host.h:6-15).
 */
#ifndef MLBM_COMPAT_H_
#define MLBM_COMPAT_H_

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#include "mlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

void mlbm_compat_set_domain(int32_t nx, int32_t ny, int32_t nz);
/* Storage of the lattice the next initialization creates (default F32). */
void mlbm_compat_set_storage(int32_t storage);

void transfer_parameter(float* tau, float* G, bool* carn_star, float* T_Tc,
                        float* rhol_spinodal, float* rhog_spinodal,
                        bool* inject_density, size_t* rho_inject_period,
                        float* rho_increment, float* rhos,
                        float* inject_position, size_t* statPeriod);

void multiphaselbm_initialization(void* rho_dd, void* psi_dd,
                                  void* pressure_dd, void* is_fluid_dd,
                                  void* collision_f_dd, void* stream_f_dd,
                                  void* force_dd);

void multiphaselbm_iteration(long step, size_t statPeriod, int reverse,
                             unsigned int inject_type);

/* The lattice behind the entry points (NULL before initialization), and its
 * release. */
mlbm_lattice* mlbm_compat_lattice(void);
void mlbm_compat_release(void);
/* Prints and exits on a CUDA error, like the reference's cudaErrorCheck. */
void mlbm_compat_check(int cuda_error, const char* file, int line);

#ifdef __cplusplus
}
#endif

#if defined(__cplusplus) && defined(lx) && defined(ly) && defined(lz)
/* The including code compiles its lattice size in: hand it over. */
#define transfer_parameter(...) \
  (mlbm_compat_set_domain(lx, ly, lz), transfer_parameter(__VA_ARGS__))
#endif

#endif /* MLBM_COMPAT_H_ */
