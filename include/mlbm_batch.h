/*
 * mlbm_batch.h -- many independent porous domains of uneven size advanced
 * together on one GPU (no counterpart in the reference, which runs one
 * compile-time-sized domain per process).
 *
 * A batch owns one mlbm_lattice per domain (same storage format, each with
 * its own size, parameters, AA phase and step origin).  mlbm_batch_iterate
 * advances every domain with one density launch and one update launch per
 * step over all domains, replayed through a CUDA graph: with FP32 / FP16
 * storage the domains live in the fluid-only (compact) layout and the
 * launches run one thread per fluid node or node pair of every domain; with
 * FP64 storage (or a domain beyond the compact kernels' limits) persistent
 * launches walk a work list of tiles of the dense layout.  Results are
 * bit-identical to the same domain advanced alone with mlbm_iterate.
 * Domains can be added and removed between iterate calls (continuous
 * batching).
 */
#ifndef MLBM_BATCH_H_
#define MLBM_BATCH_H_

#include <stdint.h>

#include "mlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mlbm_batch mlbm_batch;

mlbm_status mlbm_batch_create(int32_t storage, int32_t device,
                              mlbm_batch** out);
mlbm_status mlbm_batch_destroy(mlbm_batch* b);

/* Add a domain (host arrays in the reference layout [x][y][z]); it is
 * created, uploaded and initialised, and joins at the next iterate call with
 * its own step counter starting at step0.  *id receives its slot. */
mlbm_status mlbm_batch_add(mlbm_batch* b, int32_t nx, int32_t ny, int32_t nz,
                           const mlbm_params* params, const uint8_t* is_fluid,
                           const float* rho, int64_t step0, int32_t* id);
/* Add a domain from a checkpoint image (mlbm_checkpoint_save of a domain's
 * lattice, or of any lattice of the batch's storage): it resumes where the
 * image was taken, bit for bit, with the image's step counter.  Used to
 * preempt a domain (save, remove) and resume it later. */
mlbm_status mlbm_batch_add_checkpoint(mlbm_batch* b, const void* image,
                                      uint64_t bytes, int32_t* id);
/* Remove a domain and free its memory. */
mlbm_status mlbm_batch_remove(mlbm_batch* b, int32_t id);
/* Number of domains, and device bytes they hold. */
int32_t mlbm_batch_count(const mlbm_batch* b);
uint64_t mlbm_batch_bytes(const mlbm_batch* b);

/* Advance every domain by nsteps (asynchronous on the batch's stream). */
mlbm_status mlbm_batch_iterate(mlbm_batch* b, int32_t nsteps, int32_t reverse,
                               uint32_t inject_type);
/* The lattice of a domain: use mlbm_download_field / mlbm_phase_stats on it
 * (they run on the batch's stream and synchronise). */
mlbm_lattice* mlbm_batch_lattice(mlbm_batch* b, int32_t id);
/* Steps a domain has been advanced (its step counter). */
int64_t mlbm_batch_domain_step(const mlbm_batch* b, int32_t id);
mlbm_status mlbm_batch_synchronize(mlbm_batch* b);

/* Work-item shape of the dense mode: tile rows of the density and update
 * items, planes per update item, blocks per SM (0 = as many as fit); CUDA
 * graphs on/off (both modes). */
mlbm_status mlbm_batch_set_tuning(mlbm_batch* b, int32_t rows_density,
                                  int32_t rows_update, int32_t planes,
                                  int32_t blocks_per_sm, int32_t use_graphs);
/* Time candidate shapes on the current domains and keep the fastest (dense
 * mode; the compact mode has no shape to tune and runs no trial steps).  The
 * trial steps are real steps: every domain advances by them.  out (optional,
 * 4 ints) receives rows_density, rows_update, planes, blocks_per_sm. */
mlbm_status mlbm_batch_autotune(mlbm_batch* b, int32_t trial_steps,
                                int32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* MLBM_BATCH_H_ */
