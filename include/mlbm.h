/*
 * mlbm.h -- C ABI of the B200 D3Q19 Shan-Chen multiphase LBM library
 * (libmlbm.so).  Plain pointers, sizes and status codes; no C++ or torch types.
 *
 * One handle (mlbm_lattice) is one porous domain resident on one GPU.  The
 * calls map onto the reference's host<->device boundary
 * (include/iteration_host.h:30-60, src/iteration_host.cu:16-81 of
 * Amber1995/multiphase_LBM):
 *
 *   reference                              this ABI
 *   ------------------------------------   -----------------------------------
 *   transfer_parameter(...)                mlbm_set_params
 *     include/iteration_host.h:30-41
 *   multiphaselbm_initialization(...)      mlbm_upload_fluid_mask +
 *     include/iteration_host.h:43-49         mlbm_upload_rho + mlbm_initialize
 *   multiphaselbm_iteration(step, ...)     mlbm_iterate (n steps per call)
 *     include/iteration_host.h:56-57
 *   host reads of managed rho/pressure     mlbm_download_field
 *     src/multiphase_lbm.cu:249-252
 *   calc_cluster phase statistics          mlbm_phase_stats
 *     src/multiphase_lbm.cu:240-316
 *
 * Differences from the reference boundary, all deliberate:
 *   - lattice sizes are runtime arguments (the reference compiles them in,
 *     include/lbm_model.cuh:4-6);
 *   - every call returns an mlbm_status instead of exit()ing
 *     (include/iteration_host.h:6-15); mlbm_last_error() has the message;
 *   - fields are copied in and out in the reference's [x][y][z] layout
 *     (z fastest) instead of being shared as managed memory, so a host read
 *     never races a running kernel.
 * The three reference entry points themselves, with their own signatures,
 * are in mlbm_compat.h.
 */
#ifndef MLBM_H_
#define MLBM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLBM_ABI_VERSION 1

typedef enum mlbm_status {
  MLBM_OK = 0,
  MLBM_ERR_ARG = 1,      /* invalid argument (null, size, enum) */
  MLBM_ERR_CUDA = 2,     /* CUDA runtime error or no usable device */
  MLBM_ERR_NOMEM = 3,    /* device allocation refused */
  MLBM_ERR_STATE = 4,    /* call out of order (e.g. iterate before init) */
  MLBM_ERR_TIMEOUT = 5,  /* a bounded device wait ran out */
  MLBM_ERR_IO = 6,       /* file could not be read or written */
  MLBM_ERR_PARSE = 7     /* malformed input file */
} mlbm_status;

/* Population storage format. */
typedef enum mlbm_storage {
  MLBM_STORE_F32 = 0, /* float populations, float arithmetic (the drop-in) */
  MLBM_STORE_F16 = 1, /* half(f_i - t_i * rho_shift), float arithmetic */
  MLBM_STORE_F64 = 2  /* double populations and arithmetic (FP64 oracle) */
} mlbm_storage;

/* Fields for mlbm_download_field (reference layout [x][y][z], z fastest). */
typedef enum mlbm_field {
  MLBM_FIELD_RHO = 0,      /* density (fluid: last step's rho; solid: rhos) */
  MLBM_FIELD_PRESSURE = 1, /* EOS pressure of rho */
  MLBM_FIELD_PSI = 2,      /* pseudopotential psi(rho) */
  MLBM_FIELD_VELOCITY = 3, /* u = (sum f e + tau F)/rho, [x][y][z][3]; written
                              by the last step of an mlbm_iterate call made
                              with MLBM_ITER_WRITE_VELOCITY */
  MLBM_FIELD_POPULATIONS = 4, /* post-collision f*, [x][y][z][19] */
  MLBM_FIELD_FLUID = 5        /* solid mask as uint8 (1 = fluid) */
} mlbm_field;

typedef enum mlbm_dtype { MLBM_DTYPE_F32 = 0, MLBM_DTYPE_F64 = 1,
                          MLBM_DTYPE_U8 = 2 } mlbm_dtype;

/* Flags for mlbm_iterate. */
#define MLBM_ITER_WRITE_VELOCITY 1u

/* Physics parameters: the arguments of the reference's transfer_parameter
 * (include/iteration_host.h:30-41, defaults src/multiphase_lbm.cu:35-80) plus
 * the drainage boundary, which the reference does not have: fluid nodes with
 * x < inlet_width are held at rho_inlet and fluid nodes with
 * x >= nx - outlet_width at rho_outlet (density fixed, post-collision
 * populations the rest equilibrium t_i * rho).  Both widths 0 = periodic. */
typedef struct mlbm_params {
  float tau;
  float G;
  float T_Tc;
  float rhol_spinodal;
  float rhog_spinodal;
  float rho_increment;
  float rhos;
  float inject_position;
  int32_t carn_star;
  int32_t inject_density;
  uint64_t rho_inject_period; /* 0 = never inject */
  uint64_t stat_period;
  int32_t inlet_width;
  int32_t outlet_width;
  float rho_inlet;
  float rho_outlet;
  float rho_shift; /* FP16 storage only: populations stored minus t_i*rho_shift */
  int32_t reserved;
} mlbm_params;

/* Phase statistics over fluid nodes (calc_cluster, src/multiphase_lbm.cu:
 * 240-316; min/max of write_stats, :1057-1072).  Liquid: rho > rhol_spinodal;
 * vapour: rho < rhog_spinodal.  Sums and averages are accumulated in FP64. */
typedef struct mlbm_stats {
  int64_t n_fluid;
  int64_t n_liquid;
  int64_t n_vapour;
  int64_t n_liquid_solid_boundary;
  int64_t n_liquid_vapour_boundary;
  double mass; /* sum of rho over fluid nodes */
  double sum_p_liquid, sum_p_vapour, sum_rho_liquid, sum_rho_vapour;
  double saturation;
  double avg_p_liquid, avg_p_vapour, suction;
  double avg_rho_liquid, avg_rho_vapour;
  double ratio_liquid_solid_boundary, ratio_liquid_vapour_boundary;
  double min_rho, max_rho, min_p, max_p;
} mlbm_stats;

typedef struct mlbm_lattice mlbm_lattice;

/* Library version / diagnostics. */
int32_t mlbm_abi_version(void);
const char* mlbm_status_string(int32_t status);
/* Message of the last failing call on this host thread ("" if none). */
const char* mlbm_last_error(void);
/* D3Q19 tables as the kernels use them: e[19*3] (ex,ey,ez per direction),
 * w[19] (include/lbm_model.cuh:35-54). */
void mlbm_d3q19(int32_t* e, float* w);

/* Create a lattice of nx*ny*nz nodes on `device` with the given storage.
 * Allocates all device memory up front (MLBM_ERR_NOMEM if refused). */
mlbm_status mlbm_lattice_create(int32_t nx, int32_t ny, int32_t nz,
                                int32_t storage, int32_t device,
                                mlbm_lattice** out);
mlbm_status mlbm_lattice_destroy(mlbm_lattice* lat);
/* Device bytes held by a lattice of this size and storage (no allocation). */
uint64_t mlbm_lattice_bytes(int32_t nx, int32_t ny, int32_t nz,
                            int32_t storage);

/* CUDA stream (cudaStream_t) the lattice's work is issued on; NULL = the
 * legacy default stream. */
mlbm_status mlbm_set_stream(mlbm_lattice* lat, void* stream);

/* transfer_parameter */
mlbm_status mlbm_set_params(mlbm_lattice* lat, const mlbm_params* p);

/* Geometry and initial density, host arrays in the reference layout
 * [x][y][z] (z fastest): is_fluid (nonzero = fluid) and rho (float). */
mlbm_status mlbm_upload_fluid_mask(mlbm_lattice* lat, const uint8_t* is_fluid);
mlbm_status mlbm_upload_rho(mlbm_lattice* lat, const float* rho);
/* Same, from device memory (same layout). */
mlbm_status mlbm_upload_fluid_mask_device(mlbm_lattice* lat,
                                          const uint8_t* is_fluid_dev);
mlbm_status mlbm_upload_rho_device(mlbm_lattice* lat, const float* rho_dev);

/* multiphaselbm_initialization: f_i = t_i rho everywhere, solids take
 * rho = rhos (include/iteration_kernel.cuh:9-29).  Needs params, mask, rho. */
mlbm_status mlbm_initialize(mlbm_lattice* lat);

/* multiphaselbm_iteration for steps step0 .. step0+nsteps-1 (streaming,
 * bounce-back, Shan-Chen force, velocity shift, BGK).  Asynchronous on the
 * lattice's stream. */
mlbm_status mlbm_iterate(mlbm_lattice* lat, int64_t step0, int32_t nsteps,
                         int32_t reverse, uint32_t inject_type,
                         uint32_t flags);

/* Which kernels advance the lattice:
 *   TWO_PASS     a density launch and an update launch per step over the
 *                dense layout; bit-identical to the reference's kernels;
 *   COMPACT      the two passes over a fluid-only population layout (solid
 *                nodes own no population storage), one thread per fluid
 *                node pair (one per node in the gather step's density
 *                pass), each launch overlapping the end of the one before
 *                (programmatic dependent launch); bit-identical to
 *                TWO_PASS.  FP32 / FP16 storage, at most 2048 x 2048 x 1024
 *                nodes;
 *   BAND         ONE launch per step over the fluid-only layout with two
 *                population buffers: the launch reads the step's
 *                populations from one buffer and pushes the new ones into
 *                the other, so no block waits for another; in each block,
 *                density warps form psi of a band of rows (plus one halo
 *                row on either side) in shared memory plane by plane, and
 *                update warps follow a few planes behind, so DRAM sees the
 *                populations about once per step.  Bit-identical to
 *                TWO_PASS; FP32 / FP16 storage, whole lattices (not slabs),
 *                same size limits as COMPACT; a second population buffer is
 *                allocated on first use.  Where even a band of one row does
 *                not fit shared memory (very long rows), the steps run as
 *                COMPACT;
 *   AUTO         (default) COMPACT where supported, else TWO_PASS.
 * (Values 1, 4 and 5 belonged to step kernels this library no longer has;
 * they are refused.)  The state moves between the layouts on demand (the
 * dense buffers stay allocated; the fluid-only layout adds 19 populations
 * and 8 bytes of node table per fluid node, allocated on first use). */
#define MLBM_KERNEL_AUTO 0
#define MLBM_KERNEL_TWO_PASS 2
#define MLBM_KERNEL_COMPACT 3
#define MLBM_KERNEL_BAND 6
mlbm_status mlbm_set_step_kernel(mlbm_lattice* lat, int32_t kind);
/* The kernel the next mlbm_iterate runs (AUTO resolved); -1 for NULL. */
int32_t mlbm_get_step_kernel(const mlbm_lattice* lat);
/* Tiling of the BAND step: bands of at most `rows` rows (y, 1..64; fewer
 * where the staged rows would not fit shared memory) and chunks of about
 * `planes` planes (z, 1..1024), one block per band and chunk.  Default
 * 4 x 24. */
mlbm_status mlbm_set_band_shape(mlbm_lattice* lat, int32_t rows,
                                int32_t planes);
/* Shape of the two-pass update kernel: tile rows (block = 32 x rows
 * threads, 1..8) and planes walked per block (1..1024).  Default 4 x 16. */
mlbm_status mlbm_set_update_shape(mlbm_lattice* lat, int32_t rows,
                                  int32_t planes);
/* Time candidate shapes of the lattice's step kernel (update shape for
 * TWO_PASS, rows x planes for BAND; COMPACT has none: out = {0, 0}, no
 * steps) and keep the fastest.  The trial steps are
 * real steps (step0, step0+1, ...): the lattice advances by *steps_done of
 * them.  out (optional, 2 ints) receives rows, planes. */
mlbm_status mlbm_autotune(mlbm_lattice* lat, int64_t step0,
                          int32_t trial_steps, int32_t* out,
                          int32_t* steps_done);
/* Limit of the step kernels' bounded device waits (hand-overs between the
 * warps of one block in the BAND step), in nanoseconds; 0 = the default,
 * one second.  A wait that runs out ends the launch with the device error
 * flag set: mlbm_synchronize then reports MLBM_ERR_TIMEOUT. */
mlbm_status mlbm_set_wait_limit(mlbm_lattice* lat, uint64_t ns);
/* Testing the wait limit: the next BAND step launch makes one block wait on
 * a barrier that nothing completes, so the limit runs out (MLBM_ERR_STATE
 * for other step kernels).  The lattice must be initialised again after. */
mlbm_status mlbm_test_stall_wait(mlbm_lattice* lat);
/* Wait for the lattice's stream and report a device-side failure (a bounded
 * wait of a step kernel that ran out: MLBM_ERR_TIMEOUT; the
 * lattice must then be initialised again). */
mlbm_status mlbm_synchronize(mlbm_lattice* lat);

/* Copy a field out in the reference layout.  dtype: MLBM_DTYPE_F32 or
 * MLBM_DTYPE_F64 (F64 keeps an FP64 lattice's full precision), U8 for
 * MLBM_FIELD_FLUID.  host_out: nx*ny*nz*components elements.  Synchronous. */
mlbm_status mlbm_download_field(mlbm_lattice* lat, int32_t field,
                                int32_t dtype, void* host_out);
/* Same into device memory (stream-ordered, no synchronisation). */
mlbm_status mlbm_download_field_device(mlbm_lattice* lat, int32_t field,
                                       int32_t dtype, void* dev_out);

/* Phase statistics of the current state (device reduction, deterministic).
 * Synchronous. */
mlbm_status mlbm_phase_stats(mlbm_lattice* lat, mlbm_stats* out);
/* The same statistics without waiting, for a host loop that reads every
 * step's statistics while the next step already runs: enqueues the reduction
 * on the lattice's stream and an asynchronous copy of MLBM_STATS_RAW_LEN
 * doubles into `raw` (host memory; page-locked, or the copy waits).  Once
 * the stream has passed the call (an event recorded after it, or
 * mlbm_synchronize), mlbm_stats_from_raw gives the mlbm_stats that
 * mlbm_phase_stats would have returned at that point of the stream, and
 * reports a device error the step kernels flagged.  Calls in flight share
 * one device scratch area in stream order, so any number may be queued. */
#define MLBM_STATS_RAW_LEN 15
mlbm_status mlbm_phase_stats_async(mlbm_lattice* lat, double* raw);
mlbm_status mlbm_stats_from_raw(mlbm_lattice* lat, const double* raw,
                                mlbm_stats* out);
/* The bulk columns of the same statistics, the same way (asynchronous, raw
 * buffer of MLBM_STATS_RAW_LEN doubles, read with mlbm_stats_from_raw):
 * n_fluid, n_liquid, n_vapour, mass, the liquid and vapour density sums and
 * averages, saturation, min_rho and max_rho, each bit-identical to
 * mlbm_phase_stats.  The boundary counts and everything made of pressures
 * are not computed and read 0.  For a loop that reads the saturation and the
 * mass of every step: it skips the 18-neighbour boundary test. */
mlbm_status mlbm_bulk_stats_async(mlbm_lattice* lat, double* raw);
/* Per-x-plane counts of fluid and liquid nodes (int64[nx] each).  Sync. */
mlbm_status mlbm_plane_profile(mlbm_lattice* lat, int64_t* n_fluid_x,
                               int64_t* n_liquid_x);

/* ---- Exact checkpoints --------------------------------------------------------
 * The whole state of a lattice in its stored precision: populations (FP32,
 * FP16 bits or FP64, every node, dense layout), AA phase, density field,
 * fluid mask and parameters, plus the caller's step counter, with a
 * versioned header and a hash of the payload.  Loading an image into a
 * lattice of the same size and storage and stepping on gives, bit for bit,
 * what the saved lattice gives.  Replaces the reference's read_densities
 * resume (src/multiphase_lbm.cu:112-132), which reloads a "%.4e" density
 * field and restarts the populations from equilibrium.
 *   mlbm_checkpoint_bytes  size of the image of `lat` (header included);
 *   mlbm_checkpoint_save   write the image to host memory `image` (pinned or
 *                          pageable, at least that many bytes); synchronises
 *                          the lattice's stream;
 *   mlbm_checkpoint_load   restore params, mask, density and populations
 *                          from an image (MLBM_ERR_ARG: not an image, other
 *                          size or storage, truncated, hash mismatch);
 *                          *step (optional) receives the saved counter;
 *   mlbm_checkpoint_write / _read   the same through a file.
 * Slab lattices are refused (MLBM_ERR_STATE). */
mlbm_status mlbm_checkpoint_bytes(const mlbm_lattice* lat, uint64_t* bytes);
/* Lattice size (dims[3] = lx, ly, lz), storage and step counter of an image
 * (any of the outputs may be NULL). */
mlbm_status mlbm_checkpoint_info(const void* image, uint64_t bytes,
                                 int32_t* dims, int32_t* storage,
                                 int64_t* step);
mlbm_status mlbm_checkpoint_save(mlbm_lattice* lat, int64_t step, void* image,
                                 uint64_t bytes);
mlbm_status mlbm_checkpoint_load(mlbm_lattice* lat, const void* image,
                                 uint64_t bytes, int64_t* step);
mlbm_status mlbm_checkpoint_write(mlbm_lattice* lat, int64_t step,
                                  const char* path);
mlbm_status mlbm_checkpoint_read(mlbm_lattice* lat, const char* path,
                                 int64_t* step);

/* Phase statistics without any allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc when they need
 * statistics (an application that reserves the GPU's memory up front for its
 * own pool, or a host that forbids libraries to allocate because cudaMalloc
 * may synchronise the device and take unbounded time).  Same results as
 * mlbm_phase_stats, computed
 * from fields the caller owns: rho_dev (float) and is_fluid_dev (uint8,
 * nonzero = fluid), both device arrays in the reference layout [x][y][z]
 * (z fastest); the EOS and thresholds come from *params.  Runs on `stream`
 * (NULL = legacy default) and waits for it; *out is host memory.
 * Its scratch is a fixed static device array (about 459 KB on every GPU that
 * loads the library, kept until exit), so nx may not exceed
 * MLBM_NOALLOC_MAX_LX (MLBM_ERR_ARG otherwise).  The first call on each
 * device looks up the array's device address with cudaGetSymbolAddress,
 * which may load the library's device code on that device; a caller that
 * restricts which CUDA calls may run at a given point makes that first call
 * during its setup.  Make no call on a device after cudaDeviceReset (the
 * kept address belongs to the reset context).  Calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller. */
#define MLBM_NOALLOC_MAX_LX 4096
mlbm_status mlbm_phase_stats_noalloc(const float* rho_dev,
                                     const uint8_t* is_fluid_dev, int32_t nx,
                                     int32_t ny, int32_t nz,
                                     const mlbm_params* params, void* stream,
                                     mlbm_stats* out);

/* ---- Slab decomposition (one lattice over several GPUs) --------------------
 * A lattice of nz planes split along z into slabs, one per GPU: a slab
 * lattice of z-extent m + 2 holds the planes [z0 - 1, z0 + m] of the whole
 * lattice (periodic in z), whose first and last planes are HALO planes: the
 * step reads them but only advances the m own planes between them.  The
 * reference has no multi-GPU path; this replaces nothing in it and keeps its
 * step bit for bit: a decomposed run gives the undecomposed lattice's state
 * exactly.  Compact two-pass step only (FP32 / FP16 storage).
 *
 * Per time step, with the AA phase p of the stored state (mlbm_lattice_info):
 *   if p == 0: halo planes <- neighbours' edge planes   (MLBM_HALO_POP_*)
 *   mlbm_step_pass(lat, step, 0, ...)                    density pass
 *   psi halo planes <- neighbours' psi edge planes        (MLBM_HALO_PSI_*)
 *   mlbm_step_pass(lat, step, 1, ...)                    update pass
 *   if p == 0: neighbours' edge planes <- halo planes    (MLBM_HALO_POP_*)
 * Side 0 is the lower face (local z = 0 / 1), side 1 the upper one; the
 * EDGE segments of side 0 of one slab pair with the GHOST segments of side 1
 * of the slab below it (and side 1 with side 0 of the slab above), segment
 * for segment, equal sizes. */
#define MLBM_HALO_PSI_EDGE 0  /* psi of the own plane next to the face */
#define MLBM_HALO_PSI_GHOST 1 /* psi of the halo plane */
#define MLBM_HALO_POP_EDGE 2  /* the 5 populations of the own edge plane that
                                 the neighbour's nodes stream through */
#define MLBM_HALO_POP_GHOST 3 /* the same 5 populations of the halo plane */
#define MLBM_HALO_MAX_SEGMENTS 5

/* Mark the lattice as a slab (enable = 1; its z-extent must be >= 3) or as
 * a whole periodic lattice (0).  Call after mlbm_initialize. */
mlbm_status mlbm_set_slab(mlbm_lattice* lat, int32_t enable);
/* One pass of one time step in the current AA phase: pass 0 = density (rho
 * is written), pass 1 = update (the velocity too when flags has
 * MLBM_ITER_WRITE_VELOCITY), after which the phase flips.  step, reverse and
 * inject_type as for mlbm_iterate.  Works on any FP32/FP16 lattice; the only
 * way to step a slab lattice (mlbm_iterate refuses slabs). */
mlbm_status mlbm_step_pass(mlbm_lattice* lat, int64_t step, int32_t pass,
                           int32_t reverse, uint32_t inject_type,
                           uint32_t flags);
/* Device segments of one halo kind on one side: *count (<=
 * MLBM_HALO_MAX_SEGMENTS) pointers and byte sizes, on the lattice's device.
 * Valid until the lattice is destroyed, its mask changes or another step
 * kernel runs.  Copy them on the lattice's stream, or synchronise it first. */
mlbm_status mlbm_halo_segments(mlbm_lattice* lat, int32_t kind, int32_t side,
                               void** ptrs, int64_t* bytes, int32_t* count);

/* The halo moves among slabs held by one process as ONE kernel per
 * exchange: `ring` lists the slabs in z order (periodic); every slab's memory
 * must be reachable from the device of slabs[0], which runs the kernel (the
 * same device, or devices with peer access, which create enables).  The
 * exchange waits for every slab's stream and every slab's stream waits for
 * it.  what: MLBM_RING_POP_IN (before an AA phase-0 step), MLBM_RING_PSI
 * (between the passes), MLBM_RING_POP_OUT (after a phase-0 update; merges
 * each received slot only where its pusher is fluid).  The ring holds raw
 * device addresses of its slabs: destroy it before any of them, and build a
 * new one after a slab's mask changes. */
typedef struct mlbm_slab_ring mlbm_slab_ring;
#define MLBM_RING_POP_IN 0
#define MLBM_RING_PSI 1
#define MLBM_RING_POP_OUT 2
mlbm_status mlbm_slab_ring_create(mlbm_lattice* const* slabs, int32_t n,
                                  mlbm_slab_ring** out);
mlbm_status mlbm_slab_ring_exchange(mlbm_slab_ring* ring, int32_t what);
mlbm_status mlbm_slab_ring_destroy(mlbm_slab_ring* ring);

/* Information about the lattice: dims[3], storage, phase of the stored
 * state (0/1, see kernels), initialised flag. */
mlbm_status mlbm_lattice_info(const mlbm_lattice* lat, int32_t* dims,
                              int32_t* storage, int32_t* phase,
                              int32_t* initialized);

#ifdef __cplusplus
}
#endif

#endif /* MLBM_H_ */
