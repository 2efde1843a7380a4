/*
 * mlbm_host.h -- host-side driver surface of libmlbm: geometry, initial
 * density, command files, statistics output.  Plain C ABI; all arrays are in
 * the reference layout [x][y][z] (z fastest).  None of these calls touches
 * the GPU.
 *
 * Reference counterparts (Amber1995/multiphase_LBM):
 *   mlbm_place_sphere        MultiphaseLBM::place_sphere, src/multiphase_lbm.cu:893-927
 *   mlbm_read_positions      MultiphaseLBM::read_positions, :1106-1126
 *   mlbm_init_density        the rand() branch of resize_gpu, :134-145
 *   mlbm_read_density_vtk    the read_densities branch of resize_gpu, :112-132
 *   mlbm_generate_packing    (new) seeded sphere packing to a porosity target;
 *                            the reference's generate_solids (:1086-1103)
 *                            draws a fixed count with rand()
 *   mlbm_generate_solids     MultiphaseLBM::generate_solids, :1086-1103
 *   mlbm_packing_density     MultiphaseLBM::calc_packing_density, :1129-1142
 */
#ifndef MLBM_HOST_H_
#define MLBM_HOST_H_

#include <stdint.h>

#include "mlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Mark the nodes of one sphere solid with the reference's voxelisation:
 * sample points start at (x-R, y-R, z-R) and advance by 1.0 in float; a point
 * strictly inside (float distance^2 < R^2) marks node floor(p + 0.5), wrapped
 * once periodically.  solid_number (optional, may be NULL) receives `id`. */
mlbm_status mlbm_place_sphere(uint8_t* is_fluid, int64_t* solid_number,
                              int32_t nx, int32_t ny, int32_t nz, float x,
                              float y, float z, float R, int64_t id);

/* Read a positions file (one value per line: x, y, z, r per grain, each
 * multiplied by `resolution`) and place every grain.  *count receives the
 * number of grains; solid ids continue from *count on entry. */
mlbm_status mlbm_read_positions(const char* path, float resolution,
                                uint8_t* is_fluid, int64_t* solid_number,
                                int32_t nx, int32_t ny, int32_t nz,
                                int64_t* count);

/* rho = rho0 * (1 + rate * (rand()/RAND_MAX - 0.5)) after srand(1), loop
 * order z, y, x (the C library's rand(), as the reference). */
mlbm_status mlbm_init_density(float* rho, int32_t nx, int32_t ny, int32_t nz,
                              float rho0, float rate);

/* Seeded packing: spheres with centres uniform in [0,nx)x[0,ny)x[0,nz) and
 * radius uniform in [rmin, rmax] (splitmix64 stream from `seed`, overlap
 * allowed) are added until the porosity is <= porosity_target or
 * max_spheres are placed.  is_fluid must be all 1 on entry (it is reset).
 * xyzr (optional, 4 floats per sphere, capacity max_spheres) receives the
 * spheres in positions-file order; *count the number placed; *porosity the
 * final porosity. */
mlbm_status mlbm_generate_packing(int32_t nx, int32_t ny, int32_t nz,
                                  float rmin, float rmax,
                                  double porosity_target, uint64_t seed,
                                  int64_t max_spheres, uint8_t* is_fluid,
                                  float* xyzr, int64_t* count,
                                  double* porosity);

/* The same packing as mlbm_generate_packing, bit for bit (same spheres,
 * same count, same mask), with the voxelisation on GPU `device`: candidate
 * spheres are voxelised in chunks, each node keeping the first sphere that
 * covers it, and a prefix count of the nodes each sphere turns solid finds
 * where the porosity target is met.  No counterpart in the reference (its
 * packings come from a positions file or from generate_solids).  Allocates
 * about 4 bytes per node of device memory for the call. */
mlbm_status mlbm_generate_packing_gpu(int32_t nx, int32_t ny, int32_t nz,
                                      float rmin, float rmax,
                                      double porosity_target, uint64_t seed,
                                      int64_t max_spheres, int32_t device,
                                      uint8_t* is_fluid, float* xyzr,
                                      int64_t* count, double* porosity);
/* The reference's generate_solids: `num` grains from the C library rand(). */
mlbm_status mlbm_generate_solids(uint8_t* is_fluid, int64_t* solid_number,
                                 int32_t nx, int32_t ny, int32_t nz,
                                 int32_t num, float rmin, float rmax,
                                 float xmin, float xmax, float ymin,
                                 float ymax, float zmin, float zmax,
                                 int64_t* count);

/* Write spheres (4 floats each) as a positions file. */
mlbm_status mlbm_write_positions(const char* path, const float* xyzr,
                                 int64_t count);

/* Fraction of solid nodes. */
double mlbm_packing_density(const uint8_t* is_fluid, int32_t nx, int32_t ny,
                            int32_t nz);

/* Read the "SCALARS Density" block of a legacy VTK file written by
 * mlbm_write_vtk (or the reference's write_vtk_ascii) into rho. */
mlbm_status mlbm_read_density_vtk(const char* path, float* rho, int32_t nx,
                                  int32_t ny, int32_t nz);

#ifdef __cplusplus
}
#endif

#endif /* MLBM_HOST_H_ */
